"""Generate golden vectors from the reference's own CUDA kernels.

Run on a GPU host after ``make -C oracle ref`` (the kernels are compiled from
the reference sources):

    python tests/golden/make_golden.py [outdir]

For each case it drives the reference kernels with oracle/ref_driver.py
(a restatement of the reference's Python driver) and stores the inputs,
the integer positions, the reference's coefficient planes and CPML vectors,
the Ez traces, the residual used and the reference-mode gradients.  The
committed .npz files under tests/golden/ were produced by this script.
"""
import importlib
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import ref_driver  # noqa: E402

fg = importlib.import_module("fast-gpr-fwi_b200")


def case(wl, dev, seed):
    kw = wl.kwargs(dev)
    er = torch.clamp(kw["er"], min=1)
    se = torch.clamp(kw["se"], min=0)
    mr = kw["mr"]
    G = ref_driver.setup(dev, kw["dx"], kw["ny"], kw["nx"], 1, kw["time_windows"], kw["source_location"],
                         kw["source_step"], kw["receiver_location"], kw["receiver_step"], kw["pmlthick"],
                         kw["source_apmlitudes"], kw["step"], er, se, mr, kw["nsrc"], kw["nrx"], kw["dt"],
                         kw["Fixedreceiver"])
    rxs, hist = ref_driver.forward(G)
    traces = rxs[:, 2].contiguous()
    rng = np.random.default_rng(seed)
    resid = torch.tensor(rng.standard_normal(traces.shape).astype(np.float32), device=dev)
    ge, gs = ref_driver.backward(G, er, se, mr, hist, resid, normalize=False)
    nx, ny = wl.nx, wl.ny
    cf = [c[:nx, :ny, 0].cpu().numpy() for c in G.coef_single]
    H_uE0a = ref_driver.Grid()
    for k in ("step", "device", "dx", "dy", "dz", "nx", "ny", "nz", "dt"):
        setattr(H_uE0a, k, getattr(G, k))
    ref_driver._coefficients(H_uE0a, er, se, mr, adjoint=True)
    uE0a = H_uE0a.coef_single[0][:nx, :ny, 0].cpu().numpy()
    pml = np.zeros((8, 0), np.float32)
    if G.pmls:
        p = G.pmls[0]
        pml = np.concatenate([t.cpu().numpy() for t in (p.ERA, p.ERB, p.ERE, p.ERF, p.HRA, p.HRB, p.HRE, p.HRF)])
    out = dict(
        nx=nx, ny=ny, shots=wl.shots, nt=G.iterations, th=wl.pml, dx=np.float32(wl.dx), dt=np.float32(G.dt),
        er=er[:, :, 0].cpu().numpy(), se=se[:, :, 0].cpu().numpy(), mr=mr[:, :, 0].cpu().numpy(),
        src=G.source[:wl.shots].cpu().numpy(), rx=G.receiver[:wl.shots].cpu().numpy(),
        waveform=G.waveform.cpu().numpy(),
        uE0=cf[0], uE1=cf[1], uE4=cf[2], uH1=cf[4], uH4=cf[5], uE0a=uE0a, pml=pml,
        traces=traces.cpu().numpy(), resid=resid.cpu().numpy(),
        ge=ge[:, :, 0].cpu().numpy(), gs=gs[:, :, 0].cpu().numpy(),
    )
    return out


def main():
    outdir = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))
    os.makedirs(outdir, exist_ok=True)
    dev = torch.device("cuda:0")
    cases = {
        "small": (fg.workloads.small(), 11),
        "small_moving": (fg.workloads.small(seed=3, shots=2, nt=150, nx=40, ny=56, pml=5, nrx=6), 12),
        "config0": (fg.workloads.config0(), 13),
    }
    for name, (wl, seed) in cases.items():
        d = case(wl, dev, seed)
        np.savez_compressed(os.path.join(outdir, "ref_%s.npz" % name), **d)
        print(name, "nt", d["nt"], "max|trace|", float(np.abs(d["traces"]).max()))


if __name__ == "__main__":
    main()
