# Solvers.jl (drop-in for src/Solvers.jl, 2D) -- solve_step1..7 with the
# reference's signatures (src/Solvers.jl:14,144,242,267,344,431,459), each a
# call into libvsav on the device state.  Scalar results are Float64s; field
# results are DeviceViews (vsav_core.jl), valid until the state advances.
#
# A time step in the reference's own words (src/simulation.jl:79-110):
#     present.dt = Dt[n+1] - Dt[n]; bdf = bdf_coeff(n)
#     s1 = solve_step1(present, old, ops, conf, bdf, cache)
#     s2 = solve_step2(present, old, ops, conf, s1, bdf)
#     s3 = solve_step3(s1, s2)
#     s4 = solve_step4(present, old, ops, conf, bdf)
#     Q  = solve_step5(present, old, ops, conf, s3, s4, bdf)
#     s6 = solve_step6(s2, s3, s4, Q)
#     s7 = solve_step7(present, ops, conf, s6, bdf)
#     advance_state!(ops)          # replaces update_state!, the six assignments and the six irffts
#     download_state!(present, ops, VSAV_PRESENT)   # only when the host needs the fields

"""Step 1: the split φ/μ/ψ/ν systems, with the three ψ solves by the
diagonal-preconditioned BiCGSTAB (src/Solvers.jl:39-81).  Returns the
Step1Cache (16 device views); the `cache` argument is accepted for the
reference's signature and not written."""
function solve_step1(present, old, ops::Operators, conf, bdf::BDFCoeff, cache)
    step1!(present, ops, present.dt, bdf)
    return Step1Cache(ops, step1_views(ops))
end

"""Step 2: the two 3×3 systems for the SAV scalars; returns
(R_11_np1, R_21_np1, R_31_np1, R_12_np1, R_22_np1, R_32_np1)."""
solve_step2(present, old, ops::Operators, conf, cache, bdf::BDFCoeff) = step2_result(ops, bdf)

"""Step 3: the split fields combined with the R values (device views)."""
solve_step3(cache::Step1Cache, step2_res::NamedTuple) = step3_result(cache.ops)

"""Step 4: the two intermediate velocities ũ₁, ũ₂ (spectral and physical views)."""
solve_step4(present, old, ops::Operators, conf, bdf::BDFCoeff) = step4_result(ops, bdf)

"""Step 5: the scalar Q^{n+1} (a Float64)."""
solve_step5(present, old, ops::Operators, conf, step3_res::NamedTuple, step4_res::NamedTuple, bdf::BDFCoeff) =
    step5_result(ops, bdf)

"""Step 6: the new φ̂, ψ̂, μ̂, ν̂ (views), R1..R3 and ũ = ũ₁ + Q ũ₂."""
solve_step6(step2_res::NamedTuple, step3_res::NamedTuple, step4_res::NamedTuple, Q_np1::Float64) =
    step6_result(step3_res.ops, step4_res, Q_np1)

"""Step 7: the rotational incremental projection; the new û and p̂ (views)."""
solve_step7(present, ops::Operators, conf, step6_res::NamedTuple, bdf::BDFCoeff) = step7_result(ops, bdf)
