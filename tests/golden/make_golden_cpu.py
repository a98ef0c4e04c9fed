"""Golden vectors for the TV regulariser and the multiscale FIR filter,
produced by the reference's own Python code.

The reference's src/tv.py and src/multiscale.py import only torch, so they
run on the CPU; this script loads them by file path from the reference tree
(it is only run where that tree exists) and stores inputs and outputs:

    python tests/golden/make_golden_cpu.py [/path/to/reference] [outdir]
"""
import importlib.util
import os
import sys

import numpy as np
import torch

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FASTGPR_REFERENCE", "/root/reference")
OUT = sys.argv[2] if len(sys.argv) > 2 else os.path.dirname(os.path.abspath(__file__))


def load(name):
    spec = importlib.util.spec_from_file_location("ref_" + name, os.path.join(REF, "src", name + ".py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main():
    tv = load("tv")
    ms = load("multiscale")
    rng = np.random.default_rng(2024)
    out = {}
    # TV on a smooth layered model with noise (float32) and on a float64 model,
    # the dtype the reference notebook passes.
    z = np.linspace(0, 1, 48)[:, None]
    x = np.linspace(0, 1, 36)[None, :]
    m = 4 + 3 * (z > 0.4 + 0.1 * x) + 2 * np.exp(-((z - 0.7) ** 2 + (x - 0.5) ** 2) / 0.01)
    m32 = (m + 0.3 * rng.standard_normal(m.shape)).astype(np.float32)[:, :, None]
    out["tv_in32"] = m32
    out["tv_out32"] = tv.total_variation(torch.tensor(m32).clone()).numpy()
    m64 = (m + 0.3 * rng.standard_normal(m.shape))[:, :, None]
    out["tv_in64"] = m64
    out["tv_out64"] = tv.total_variation(torch.tensor(m64).clone()).numpy()
    sig = (2e-3 + 1e-3 * rng.random((30, 20))).astype(np.float32)[:, :, None]
    out["tv_sig_in"] = sig
    out["tv_sig_out"] = tv.total_variation(torch.tensor(sig).clone()).numpy()
    # FIR: design (odd and even tap counts) and application to 1-D and 3-D data
    for fs, fc in ((1e10, 1e8), (1e10, 2.5e8), (8e9, 1e8), (1.25e10, 2e8)):
        key = "fir_%d_%d" % (int(fs / 1e6), int(fc / 1e6))
        out[key + "_taps"] = ms.design_fir_filter(fc, fs, int(fs / fc)).numpy()
    data3 = rng.standard_normal((3, 400, 5)).astype(np.float32)
    out["fir_data3"] = data3
    out["fir_out3"] = ms.apply_filter(torch.tensor(data3), 1e10, 1e8).numpy()
    data1 = rng.standard_normal(300).astype(np.float32)
    out["fir_data1"] = data1
    out["fir_out1"] = ms.apply_filter(torch.tensor(data1), 8e9, 1e8).numpy()
    os.makedirs(OUT, exist_ok=True)
    np.savez_compressed(os.path.join(OUT, "ref_tv_fir.npz"), **out)
    print("wrote", os.path.join(OUT, "ref_tv_fir.npz"), sorted(out))


if __name__ == "__main__":
    main()
