"""CPU oracle for the implicit cpGIMP load step — TEST INFRASTRUCTURE ONLY.

This package restates, in NumPy FP64 (complex-step capable), the algorithm of
GeoWarp's implicit cpGIMP material point path:

  * cpGIMP shape functions            mpm/gimp.py:25-507
  * particle seeding / initial state  mpm/mpm_utils.py:12-81
  * P2G activation, pressure BCs,
    consistent-mass projection        mpm/mpm_utils.py:83-414
  * residual kernels                  mpm/mpm_utils.py:416-1294
  * Jacobian layout / masking         solvers/sparse_differentiation.py:213-401,
                                      mpm/mpm_utils.py:1299-1348
  * G2P and lp update                 mpm/mpm_utils.py:1351-1590, mpm/gimp.py:428-507
  * J2 return map                     materials/plasticity.py:8-37
  * Drucker-Prager return map         problems/material_tests/triaxial_DruckerPrager.py:119-412
  * NorSand return map                problems/material_tests/triaxial_NorSand.py:155-400
  * solver loops ('scipy' path)       solvers/quasi_static_solver_2d.py:144-258,
                                      solvers/quasi_static_coupled_solver_2d.py:164-313,
                                      solvers/quasi_static_coupled_solver_3d.py:206-420

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it, always as the checker.  The engine in
``geowarp_b200`` never calls into this package.

Parity status: UNPINNED against the Warp reference itself.  The reference runs
only on NVIDIA Warp (``warp-lang==1.7.0``), which is not installable in this
environment, and its tree holds no tests, fixtures or golden vectors.  The
oracle is pinned instead by the analytic known answers the reference's driver
scripts compare against (bar under self-weight, J2 bar, Terzaghi consolidation),
and its Jacobian is exact to machine precision (complex-step differentiation),
replacing Warp's coloured reverse-mode tape (solvers/sparse_differentiation.py).
"""
