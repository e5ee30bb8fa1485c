"""CPU oracle for the sparse D3Q27 lattice-Boltzmann step — TEST INFRASTRUCTURE ONLY.

Nothing in the `cerebrosim_b200` package imports this folder. Only `tests/`, `__graft_entry__.smoke()` and the
`cpu_baseline` / `--impl reference` legs of `bench.py` use it, and there only as the checker or as the timed CPU
restatement of the reference.

  lattice_ref.py  NumPy restatement of CerebroSim `lbm.build_lattice` (lbm.py:264-330), `scatter` (lbm.py:333-338),
                  `Units` (lbm.py:63-82) and `Solver.set_sponge` (lbm.py:398-416). Pinned bit-exactly against
                  tables written by the reference itself (tests/golden/).
  lbm_ref.cpp     C++ restatement of `k_clock` (lbm.py:90-102), `_ddx` / `_h3` (lbm.py:105-137), `k_step`
                  (lbm.py:140-257) and the flux / outlet-resistance kernels `k_flux` / `k_bc` (simulate.py:65-82),
                  templated on float / double, OpenMP over nodes, following the reference's order of operations.
                  Bit-level parity with the reference's compiled GPU arithmetic is unpinned (the reference's GPU
                  dialect cannot run here); the step is pinned against the reference's published validation
                  numbers (reports/step3_report.md:20-33).
  step_ref.py     ctypes wrapper + `OracleSolver`, mirroring `lbm.Solver` (lbm.py:346-455).
"""
