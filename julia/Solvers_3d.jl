# Solvers_3d.jl (drop-in for src/Solvers_3d.jl, 3D) -- solve_step1..7 with the
# reference's 3D signatures (src/Solvers_3d.jl:14,99,196,221,299,400,428).  The
# device path is the same as in 2D; Step 1 divides ψ by the constant-mobility
# symbol (src/Solvers_3d.jl:28-30) unless the handle was built with
# psi3d_variable = true, and Step 5 uses conf.dt as the reference's 3D Step 5
# does (src/Solvers_3d.jl:386-387).
include(joinpath(@__DIR__, "Solvers.jl"))
