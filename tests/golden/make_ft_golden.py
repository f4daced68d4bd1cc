"""Generate tests/golden/ft_tools_cases.npz: inputs and outputs of the
reference's own spectrogram-grid tools (ft_tools_cffi.cpp over ft_tools.hpp,
built from the reference tree into oracle/_ref/ by `make -C oracle ref`) for the grid
pipeline cases of tests/test_gpu_ft_tools.py.

    make -C oracle ref REF=<reference tree> && python tests/golden/make_ft_golden.py
"""
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, REPO)

from oracle import ft_tools as ft  # noqa: E402

# (name, polar, T, F, spec, plan, quant, contrast)
CASES = [
    ("cx_quant_contrast3", 0, 24, 33, (0.0, 0.0, 1.0, 10.0), None, (1, 55.0, 0.05, 0.5, 8.0),
     (1, 3, 3, 0.0, 0.5, 1.0, 1)),
    ("cx_resample2_gamma", 0, 20, 17, (0.0, 5.0, 1.0, 20.0), (2, 2, 2, 2, 1), (1, 110.0, 0.1, 0.7, 4.0),
     (1, 5, 3, 0.02, 0.8, 0.7, 1)),
    ("po_quant_contrast3", 1, 24, 33, (0.0, 0.0, 1.0, 10.0), None, (1, 55.0, 0.05, 0.5, 8.0),
     (1, 3, 3, 0.0, 0.5, 1.0, 1)),
    ("po_resample_freq3_global", 1, 16, 21, (0.0, 0.0, 1.0, 7.0), (1, 3, 1, 3, 0), None,
     (1, 0, 0, -0.1, 1.5, 2.0, 0)),
    ("cx_global_time", 0, 18, 40, (0.0, 0.0, 1.0, 3.0), None, None, (1, 0, 5, 0.0, 0.3, 1.0, 1)),
    ("cx_global_freq", 0, 18, 40, (0.0, 0.0, 1.0, 3.0), None, None, (1, 3, 0, 0.1, 0.3, 1.3, 1)),
    ("po_quant_nobase", 1, 12, 9, (0.0, 1.0, 1.0, 1.0), None, (1, 0.0, 0.0, 0.4, 8.0), None),
    ("cx_up3x2_down3x2", 0, 10, 12, None, (3, 2, 3, 2, 1), (1, 30.0, 0.2, 0.9, 2.0), (1, 7, 5, 0.0, 1.0, 1.0, 0)),
    ("cx_shape_mismatch", 0, 8, 8, None, (2, 1, 3, 1, 1), None, None),
    ("po_large", 1, 200, 129, (0.0, 0.0, 1.0, 43.06640625), (2, 2, 2, 2, 1), (1, 220.0, 0.01, 0.5, 6.0),
     (1, 3, 5, 0.0, 0.4, 0.8, 1)),
]


def structs(spec, plan, quant, contrast):
    return (ft.GridSpec(*spec) if spec else None, ft.ResamplePlan(*plan) if plan else None,
            ft.QuantizerConfig(*quant) if quant else None, ft.ContrastConfig(*contrast) if contrast else None)


def inputs(name, polar, T, F):
    rng = np.random.default_rng(sum(map(ord, name)))
    if polar:
        a = rng.uniform(0.0, 2.0, (T, F)).astype(np.float32)
        b = rng.uniform(-np.pi, np.pi, (T, F)).astype(np.float32)
    else:
        a = rng.standard_normal((T, F)).astype(np.float32)
        b = rng.standard_normal((T, F)).astype(np.float32)
    return a, b


def main():
    out = {}
    for name, polar, T, F, spec, plan, quant, contrast in CASES:
        a, b = inputs(name, polar, T, F)
        ok, ra, rb = ft.apply(a, b, T, F, *structs(spec, plan, quant, contrast), polar=bool(polar))
        out[name + "/a"] = a
        out[name + "/b"] = b
        out[name + "/ok"] = np.int32(ok)
        out[name + "/ra"] = ra
        out[name + "/rb"] = rb
    np.savez_compressed(os.path.join(REPO, "tests", "golden", "ft_tools_cases.npz"), **out)
    print("wrote", len(CASES), "cases")


if __name__ == "__main__":
    main()
