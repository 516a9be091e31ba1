# Utils_3d.jl (drop-in for src/Utils_3d.jl, 3D): the same functions as Utils.jl,
# which handles both ranks (the 3D f_surf keeps the reference's missing ∂z
# term, src/Utils_3d.jl:38-41).
include(joinpath(@__DIR__, "Utils.jl"))
