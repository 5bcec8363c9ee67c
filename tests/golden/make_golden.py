"""Converts the reference's self-contained golden files into the compact fixtures the oracle
tests read, so the tests run where the reference tree is absent.

Sources (physwkim/ptyrs, `ptyrs/tests/engine/data/`): the rPIE near-field set
`rpie_near_*_f64.txt` (pty-chi RPIEReconstructor in float64, written by the reference's
`refs/f64/rpie_near.py`) and the LSQML near-field set `lsqml_near_*_f64.txt` (pty-chi LSQML in
float64, `refs/f64/lsqml_near.py`), and the PyNX set `pynx_near_*_f64.txt` (PyNX `cpu_operator` promoted
to float64, `refs/f64/pynx_near.py`) whose ML run pins the Poisson conjugate gradient, and `lsqml_near_pos_*_f64.txt` (one pty-chi
LSQML step refining the positions under PATCH, `refs/f64/lsqml_near_pos.py`) and
`lsqml_multislice_*_f64.txt` (pty-chi LSQML through three slices with angular-spectrum, Fresnel
and far-field exits, `refs/f64/lsqml_multislice.py`). Each text table becomes one float64 array of the same
rows and columns under its stem in `rpie_near.npz`, `lsqml_near.npz` and `pynx_near.npz`.

    python tests/golden/make_golden.py [REFERENCE_ROOT]
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
}


def main(root):
    data = os.path.join(root, "ptyrs", "tests", "engine", "data")
    here = os.path.dirname(os.path.abspath(__file__))
    for group, stems in GROUPS.items():
        arrays = {}
        for stem in stems:
            path = os.path.join(data, f"{group}_{stem}_f64.txt")
            arrays[stem] = np.loadtxt(path, ndmin=2)
        np.savez_compressed(os.path.join(here, f"{group}.npz"), **arrays)
        print(group, {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
