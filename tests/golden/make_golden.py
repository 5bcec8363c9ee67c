"""Converts the reference's self-contained golden files into the compact fixtures the oracle
tests read, so the tests run where the reference tree is absent.

Sources (physwkim/ptyrs, `ptyrs/tests/engine/data/`): the rPIE near-field set
`rpie_near_*_f64.txt` (pty-chi RPIEReconstructor in float64, written by the reference's
`refs/f64/rpie_near.py`) and the LSQML near-field set `lsqml_near_*_f64.txt` (pty-chi LSQML in
float64, `refs/f64/lsqml_near.py`), and the PyNX set `pynx_near_*_f64.txt` (PyNX `cpu_operator` promoted
to float64, `refs/f64/pynx_near.py`) whose ML run pins the Poisson conjugate gradient, and `lsqml_near_pos_*_f64.txt` (one pty-chi
LSQML step refining the positions under PATCH, `refs/f64/lsqml_near_pos.py`) and
`lsqml_multislice_*_f64.txt` (pty-chi LSQML through three slices with angular-spectrum, Fresnel
and far-field exits, `refs/f64/lsqml_multislice.py`); and the far-field results on the seeded
scenario `dm_scenario(32, 40, nprobe, 2e5, 4.0)` (`tests/common/engine/scenario.rs`), whose
counts `oracle/scenario.py` redraws: the position gradient (`pos_grad*`), ML with positions
(`ml_pos_*`), LSQML steps and epochs with and without positions (`lsqml_*`), rPIE against
pty-chi (`rpie_ptychi_f64.txt`) and with positions under PATCH (`rpie_pos_*`), DM and RAAR
against PyNX (`dm_pynx_f64.txt`, `raar_pynx_f64.txt`), and OPR probe variation alone and inside
an LSQML step (`opr_*`, `lsqml_opr_*`, `lsqml_opr_int_*`). Each text table becomes one float64 array of the same rows and
columns under its stem (`table` for a file without one) in `<group>.npz`.

The I/O fixtures (`ptyrs/tests/io/data/`) are copied as they are: `pynx_small.cxi` (written by
PyNX's `save_ptycho_data_cxi` through libhdf5, `make_pynx_small.py` there) and
`ptypy_small_{single,double}.ptyr` (PtyPy `Ptycho.save_run`, `make_ptypy_small.py` there), the
files the library's HDF5 reader is checked on.

    python tests/golden/make_golden.py REFERENCE_ROOT [GROUP ...]
"""
import os
import sys

import numpy as np

GROUPS = {
    "rpie_near": ["cases", "corners", "counts", "obj", "probe", "runs", "llk", "run_obj",
                  "run_probe"],
    "lsqml_near": ["cases", "corners", "counts", "obj", "probe", "icalc", "llk",
                   "step_steps", "step_obj", "step_probe", "epochs_steps", "epochs_obj",
                   "epochs_probe"],
    "pynx_near": ["case", "corners", "counts", "obj", "probe", "runs", "llk", "run_obj",
                  "run_probe"],
    "lsqml_near_pos": ["start", "steps", "offsets", "obj", "probe"],
    "lsqml_multislice": ["cases", "corners", "counts", "obj", "probe", "icalc", "llk",
                         "step_steps", "step_obj", "step_probe", "epochs_steps", "epochs_obj",
                         "epochs_probe"],
    # one LSQML step through the three slices refining positions under Patch
    # (refs/f64/lsqml_multislice_pos.py): the start slices, steps, offsets and changes
    "lsqml_multislice_pos": ["start", "steps", "offsets", "obj", "probe"],
    # The far-field sets on the seeded scenario `dm_scenario(32, 40, nprobe, 2e5, 4.0)`, whose
    # counts the oracle redraws (oracle/scenario.py): results only, no state.
    "pos_grad": ["", "values"],
    "ml_pos": ["obj", "offsets", "probe"],
    "lsqml_gaussian": ["obj", "probe", "steps"],
    "lsqml_poisson": ["obj", "probe", "steps"],
    "lsqml_epochs_gaussian": ["obj", "probe", "steps"],
    "lsqml_epochs_poisson": ["obj", "probe", "steps"],
    "lsqml_pos": ["steps", "offsets", "obj", "probe"],
    "lsqml_pos_epochs": ["steps", "offsets", "obj", "probe"],
    # pty-chi BH on the amplitude cost, two epochs with one batch of every frame (conjugate
    # directions) and with batches of 16 (steepest descent); step rows padded with -1
    "bh_full": ["obj", "probe", "steps"],
    "bh_mini": ["obj", "probe", "steps"],
    # the same with the offsets refined under Patch (refs/f64/bh_pos.py; position_rho 2):
    # every frame's offsets before and after, the object and probe changes of both epochs
    "bh_pos_full": ["obj", "probe", "offsets", "steps"],
    "bh_pos_mini": ["obj", "probe", "offsets", "steps"],
    # through three slices (refs/f64/bh_multislice.py, on lsqml_multislice's state and counts;
    # probe_rho 1): per case and method the steps, the slices' and the probe's changes
    "bh_multislice": ["steps", "obj", "probe"],
    # one LSQML step refining the offsets with three eigenmodes of probe mode 0
    "lsqml_pos_opr": ["eigen", "weights", "steps", "offsets", "obj", "probe"],
    "rpie_ptychi": [""],
    "dm_pynx": [""],
    "raar_pynx": [""],
    "opr": ["eigen", "weights", "values"],
    "lsqml_opr": ["eigen", "weights", "values", "steps", "obj", "probe"],
    "lsqml_opr_int": ["eigen", "weights", "values", "steps", "obj", "probe"],
    "rpie_pos_step": ["obj", "probe", "offsets"],
    "rpie_pos_epochs": ["obj", "probe", "offsets"],
}


IO_FILES = ["pynx_small.cxi", "ptypy_small_single.ptyr", "ptypy_small_double.ptyr"]


def load_table(path):
    """A whitespace table as float64 rows; rows of unequal length (a batch's frames at the end
    of each step row) are padded with -1."""
    rows = [[float(v) for v in line.split()] for line in open(path) if line.strip()]
    width = max(len(r) for r in rows)
    return np.array([r + [-1.0] * (width - len(r)) for r in rows], np.float64).reshape(
        len(rows), width)


def main(root, only=()):
    data = os.path.join(root, "ptyrs", "tests", "engine", "data")
    here = os.path.dirname(os.path.abspath(__file__))
    for group, stems in GROUPS.items():
        if only and group not in only:
            continue
        arrays = {}
        for stem in stems:
            name = f"{group}_{stem}_f64.txt" if stem else f"{group}_f64.txt"
            arrays[stem or "table"] = load_table(os.path.join(data, name))
        np.savez_compressed(os.path.join(here, f"{group}.npz"), **arrays)
        print(group, {k: v.shape for k, v in arrays.items()})
    if not only or "io" in only:
        io = os.path.join(root, "ptyrs", "tests", "io", "data")
        for name in IO_FILES:
            with open(os.path.join(io, name), "rb") as src:
                blob = src.read()
            with open(os.path.join(here, name), "wb") as dst:
                dst.write(blob)
            print(name, len(blob), "bytes")


if __name__ == "__main__":
    # the checkout of physwkim/ptyrs whose golden tables are converted: the first argument, or
    # PTYRS_REFERENCE
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PTYRS_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py PTYRS_CHECKOUT (or set PTYRS_REFERENCE)")
    main(root, sys.argv[2:])
