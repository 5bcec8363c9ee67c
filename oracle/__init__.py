"""CPU f64 oracle for the ptychography reconstruction hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, in numpy float64, the reference engine's CPU operators for the path
that the CUDA library accelerates (physwkim/ptyrs, crate `ptyrs`, modules `base` and
`engine`): position preprocessing and the address table, the seeded mini-batches, the
observed-intensity layout, the unitary FFT and the free-space propagators, the PyNX/pty-chi
operators, and the rPIE, ML (Poisson conjugate gradient) and LSQML loops.  Every function
cites the reference file:line it follows.

Who may use it: only `tests/`, `__graft_entry__.smoke()` and the `cpu_baseline` leg of
`bench.py` (and `bench.py --impl reference`), and there only as the checker or the timed CPU
baseline.  The product path (`ptyrs_b200`) never imports it; it fails loudly when its CUDA
library is missing.

Parity pins: the oracle is checked against the reference's own self-contained golden files
(`ptyrs/tests/engine/data/rpie_near_*`, `lsqml_near_*`, converted to `tests/golden/*.npz` by
`tests/golden/make_golden.py`) and against the known-answer unit tests of
`ptyrs/src/base/{addr,positions}.rs` and `ptyrs/src/engine/{obs,ops,batch}.rs`.
"""
