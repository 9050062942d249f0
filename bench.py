#!/usr/bin/env python
"""Benchmark: batched FP64 RGF energy-points/s at b=256, L=64 on B200.

Workload (synthetic, seeded): random Hermitian tight-binding device with
block size b=256 and L=64 blocks (onsite diag U[-2,2] eV + Hermitian Gaussian
sigma=0.3/sqrt(b); couplings Gaussian sigma=1/sqrt(b); S = I + Hermitian
Gaussian sigma=0.01/sqrt(b), non-zero S couplings), 2048 energies in [-3,3] eV,
eta=1e-5, complex128.  One step = one k-realisation (its own seeded device)
over all 2048 energies: the full RGF sweep with T(E) and DOS reduced in the
same launch.  Each rank handles its own k-realisations (weak scaling, no
data-path collective).  The headline value is the plain FP64 sweep; the line
also carries the mixed-precision sweep (tcgen05 3xTF32 products), its
FP64-residual refined form with the T(E) error against the FP64 run, and the
forward+adjoint throughput of both (``mixed`` and ``adjoint`` objects; one
warm-up and one timed step each, rank 0 only).

Prints one JSON line (rank 0).  ``--impl reference`` times the CPU oracle
(numpy restatement of the reference recursive_gf + T/DOS) on the host cores
for the same workload instead.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RGF energy-points/s @ b=256,L=64: FP64 vs mixed+adjoint on 1 B200; % roofline"
UNIT = "energy-points/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--b", type=int, default=256)
    ap.add_argument("--L", type=int, default=64)
    ap.add_argument("--energies", type=int, default=2048)
    ap.add_argument("--eta", type=float, default=1e-5)
    ap.add_argument("--cpu-energies", type=int, default=0, help="CPU baseline sample size (0: one per process)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--phases", action="store_true", help="report per-phase SM-cycle shares")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision and adjoint legs")
    ap.add_argument("--refine-steps", type=int, default=3)
    ap.add_argument("--configs", default="",
                    help="extra legs, comma separated: 'uneven' (the 512-device uneven batch, 128 devices), "
                         "'leads' (its lead decimation alone, --lead-devices devices), 'scf' (b=512 SCF "
                         "loop captured as a CUDA graph), not in the default run; 'products' (the G Gamma "
                         "G^H sum, the Bloch coupling product and the lead adjoint, each timed alone) is in "
                         "the default line unless --no-products")
    ap.add_argument("--lead-devices", type=int, default=128, help="devices whose leads the 'leads' leg decimates")
    ap.add_argument("--lead-eta", type=float, default=1e-5, help="lead broadening of the 'leads' leg")
    ap.add_argument("--no-leads", action="store_true", help="skip the metric device's lead decimation object")
    ap.add_argument("--no-products", action="store_true",
                    help="skip the product-chain timings (G Gamma G^H sum, Bloch coupling, lead adjoint)")
    ap.add_argument("--uneven-devices", type=int, default=128, help="devices of the 'uneven' leg")
    ap.add_argument("--uneven-chunk", type=int, default=128, help="devices per launch in the 'uneven' leg")
    ap.add_argument("--scf-k", type=int, default=8, help="k-points of the 'scf' leg")
    ap.add_argument("--scf-energies", type=int, default=37, help="energies per k of the 'scf' leg (4096: config)")
    ap.add_argument("--scf-iters", type=int, default=10, help="timed SCF iterations of the 'scf' leg")
    ap.add_argument("--uneven-precisions", default="fp64,mixed,mixed_refined",
                    help="runs of the 'uneven' leg besides FP64: mixed, mixed_refined")
    ap.add_argument("--inverse", default=None, choices=["gj", "block"],
                    help="Schur-complement inverse: pivoted Gauss-Jordan or recursive 2x2 blocks "
                         "(default: the autotuned scheme, else block)")
    ap.add_argument("--torch-energies", type=int, default=128,
                    help="energies of the torch-on-CUDA reference-path sample (0: skip that leg)")
    return ap.parse_args()


def flops_per_point(b, L):
    """Algorithmic work of one retarded RGF energy point: 9 complex n^3 MACs per block (4M)."""
    return 72.0 * b ** 3 * L


class Clocks:
    """nvidia-smi sampler running during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_fp64_peak(torch):
    """cuBLAS DGEMM (FP64 tensor cores) 8192^3, best of 5 -- the FP64 roofline denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = a @ b
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.mm(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def measured_tf32_peak(torch):
    """cuBLAS FP32 GEMM with TF32 tensor cores 8192^3, best of 5 -- the mixed path's denominator."""
    n = 8192
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    a = torch.randn(n, n, dtype=torch.float32, device="cuda")
    b = torch.randn(n, n, dtype=torch.float32, device="cuda")
    c = a @ b
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.mm(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    torch.backends.cuda.matmul.allow_tf32 = old
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def torch_reference_tdos(hd, hu, hl, sd, su, sl, E, seL, seR, eta):
    """T(E) and DOS of a uniform-block device by the reference's own GPU algorithm, in torch.

    The reference runs recursive_gf on CUDA as torch complex128 operations:
    recursive_green_cal.py:395-463 copies the diagonal blocks (``* 1.``), adds
    the lead self-energies into the corners and stacks every block list to
    [K, B, n, n]; the stacked branch of recursive_gf_cal (:69-114) forms
    D - zS, L - zS_l, U - zS_u, solves g_0 = (-D_0)^-1 and
    g_{q+1} = (-D_{q+1} - L_q g_q U_q)^-1 with torch.linalg.solve against the
    identity, and runs the backward products with batched matmuls.  T(E) is
    DeviceProperty._cal_tc_ (device_property.py:374-406) and the DOS
    _cal_dos_ (:408-439).  This restatement issues the same torch calls on
    the same shapes, so on a GPU it times the library path (cuSOLVER / cuBLAS)
    the reference would take.  ``E`` is [B] real, ``seL``/``seR`` [B, n, n].
    """
    import torch
    K, B, n = len(hd), E.shape[0], hd[0].shape[-1]
    ex = lambda t: t.unsqueeze(0).expand(B, -1, -1)
    Dl = [ex(h) * 1. for h in hd]
    cl, cr = min(n, seL.shape[-1]), min(n, seR.shape[-1])
    Dl[0][:, :cl, :cl] = Dl[0][:, :cl, :cl] + seL[:, :cl, :cl]
    Dl[-1][:, -cr:, -cr:] = Dl[-1][:, -cr:, -cr:] + seR[:, -cr:, -cr:]
    D, L, U = torch.stack(Dl), torch.stack([ex(t) for t in hl]), torch.stack([ex(t) for t in hu])
    Sd, Sl, Su = torch.stack([ex(t) for t in sd]), torch.stack([ex(t) for t in sl]), torch.stack([ex(t) for t in su])
    z = (E.to(torch.complex128) + 1j * eta).view(1, -1, 1, 1)
    md, ml, mu = D - z * Sd, L - z * Sl, U - z * Su
    eye = torch.eye(n, dtype=md.dtype, device=md.device).expand(B, n, n)
    g = [torch.linalg.solve(-md[0], eye)]
    for q in range(K - 1):
        g.append(torch.linalg.solve(-md[q + 1] - ml[q] @ g[q] @ mu[q], eye))
    del md
    grd, grl, gru = [None] * K, [None] * (K - 1), [None] * (K - 1)
    grd[-1] = g[-1].clone()
    gt = g[-1].clone()
    for q in range(K - 2, -1, -1):
        gU = g[q] @ mu[q]
        grl[q] = grd[q + 1] @ ml[q] @ g[q]
        gru[q] = gU @ grd[q + 1]
        grd[q] = g[q] + gU @ grl[q]
        gt = gU @ gt
    gam = lambda s: 1j * (s - s.mH)
    GL = torch.zeros((B, n, n), dtype=gt.dtype, device=gt.device)
    GR = torch.zeros_like(GL)
    GL[:, :cl, :cl] += gam(seL)[:, :cl, :cl]
    GR[:, -cr:, -cr:] += gam(seR)[:, -cr:, -cr:]
    T = (GL @ gt @ GR @ gt.mH).diagonal(dim1=-2, dim2=-1).real.sum(-1)
    dos = 0
    for j in range(K):
        t = grd[j] @ sd[j]
        if j > 0:
            t = t + grl[j - 1] @ su[j - 1]
        if j < K - 1:
            t = t + gru[j] @ sl[j]
        dos = dos - t.imag.diagonal(dim1=-2, dim2=-1).sum(-1) / math.pi
    return T, 2 * dos


def torch_reference_leg(torch, dev, E, seL, seR, eta, n_energies, chunk=32):
    """Time torch_reference_tdos on the GPU: a sample of ``n_energies`` energies of the workload, in
    batches of ``chunk`` (the reference keeps K x B x n^2 stacks per call, so the energies go
    through it in batches, as its e_batch_size does); CUDA events around each pass, best of two.
    Returns (T of the sample, sample indices, milliseconds)."""
    idx = torch.linspace(0, E.shape[0] - 1, n_energies).round().long()
    Es, sL, sR = E[idx].real.cuda(), seL[idx], seR[idx]
    hd, hu, hl, sd, su, sl = ([t.cuda() for t in x] for x in (dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl))

    def run():
        Ts = []
        for a in range(0, n_energies, chunk):
            T, _ = torch_reference_tdos(hd, hu, hl, sd, su, sl, Es[a:a + chunk], sL[a:a + chunk],
                                        sR[a:a + chunk], eta)
            Ts.append(T)
        return torch.cat(Ts)

    run()  # warm-up (library handles, workspaces)
    torch.cuda.synchronize()
    ms = float("inf")
    for _ in range(2):  # best of two timed passes: the baseline's most favourable time
        a, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        T = run()
        b_.record()
        torch.cuda.synchronize()
        ms = min(ms, a.elapsed_time(b_))
    return T, idx, ms


def current_density_leg(torch, rgf_plan, workload, eta):
    """Gradient cost of the current + density loss: b=96, L=32, 1024 energies in [-0.3, 0.3] eV.

    Loss = I + n with I = sum_E w_E T(E), w_E the trapezoid weights of the Landauer window
    f_L - f_R at V = 0.3 V, kT = 25 meV, and n = sum_E v_E DOS(E), v_E = f(E) x trapezoid weight
    (the occupied part of the window).  Forward = one T + DOS sweep; gradient = the one adjoint
    launch returning T and d(I + n)/d(every H, S block, both self-energies).  Both precisions,
    one warm-up and one timed call each (CUDA events)."""
    b, L, nE = 96, 32, 1024
    d = workload.random_device(b, L, seed=4242)
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(d.hd, d.hu, d.hl, d.sd, d.su, d.sl)])
    E = torch.linspace(-0.3, 0.3, nE, dtype=torch.float64)
    seL = workload.random_self_energy(nE, b, seed=4243).cuda()
    seR = workload.random_self_energy(nE, b, seed=4244).cuda()
    dx = float(E[1] - E[0])
    tw = torch.full((nE,), dx, dtype=torch.float64)
    tw[0] = tw[-1] = dx / 2
    kT, V = 0.025, 0.3
    fL = 1 / (1 + torch.exp((E - V / 2) / kT))
    fR = 1 / (1 + torch.exp((E + V / 2) / kT))
    wI = (fL - fR) * tw
    wn = 0.5 * (fL + fR) * tw
    Ez = E.to(torch.complex128).cuda()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        a, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b_.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b_)

    out = {}
    for prec in ("fp64", "mixed"):
        tf = timed(lambda: rgf_plan.run(geom, [Ez], [seL], [seR], eta=eta, outputs=(), trans=True, dos=True,
                                        check=False, precision=prec))
        tg = timed(lambda: rgf_plan.run(geom, [Ez], [seL], [seR], eta=eta, outputs=(), check=False,
                                        adjoint_w=wI, adjoint_w_dos=wn, precision=prec))
        out[prec] = {"forward_value": nE / (tf * 1e-3), "grad_value": nE / (tg * 1e-3), "grad_over_forward": tg / tf,
                     "unit": UNIT}
        if prec == "fp64":  # the config's "checkpoints every 6 blocks": g_q kept for q = 0, 6, ... only
            tc = timed(lambda: rgf_plan.run(geom, [Ez], [seL], [seR], eta=eta, outputs=(), check=False,
                                            adjoint_w=wI, adjoint_w_dos=wn, precision=prec, checkpoint=6))
            out[prec]["checkpoint6"] = {"grad_value": nE / (tc * 1e-3), "grad_over_forward": tc / tf,
                                        "g_storage_blocks_per_slot": f"{(L + 5) // 6 + 6} of {L} (g and its "
                                                                     f"z-tangent each)"}
    out["note"] = ("config-4 loss I + n (Landauer current by trapezoid weights at V=0.3 V, kT=25 meV, plus the "
                   "occupied summed onsite density); grad_value = energy points/s of T plus the full gradient "
                   "from one adjoint launch (T adjoint + z-tangent density pass); grad_over_forward = that "
                   "launch / a T+DOS forward launch")
    return out


def _timed(torch, fn):
    """(fn(), milliseconds) with CUDA events on the current stream."""
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    r = fn()
    b.record()
    torch.cuda.synchronize()
    return r, a.elapsed_time(b)


# Lead broadening of the synthetic leads (edge blocks of random dense devices) in the opt-in legs;
# the decimation's LU solve keeps the residual check within the reference's bound at 1e-5.
ETA_LEAD_SYNTH = 1e-5


def products_leg(torch, peak, n=256, n_nodes=256, n_bloch=256, n_lead_e=64, eta=ETA_LEAD_SYNTH, seed=77):
    """The product chains beside the sweep, each timed alone through its Python API with CUDA
    events (descriptor packing and the status read included): the DM_neq sum of Ozaki.integrate
    (negf_gamma_sum_run) over n_nodes Gauss nodes of an n x n first block with an n x n Gamma_R;
    the Bloch coupling product (the decimation kernel's coupling mode) on n_bloch unfolded
    2n x 2n surface Green's functions with an n x n H_DL; the lead-parameter adjoint
    (negf_lead_adjoint_run) of the b = n metric device's left lead at n_lead_e energies.  Work is
    counted as 8 flop per complex multiply-add (4M), as for the sweep."""
    from dpnegf_b200 import products, workload
    from dpnegf_b200.surface_green import LeadArena, LeadBlocks, self_energies
    gen = torch.Generator(device="cuda").manual_seed(seed)
    rnd = lambda *s: torch.randn(*s, dtype=torch.complex128, device="cuda", generator=gen) / n ** 0.5
    res = {}

    def rec(name, ms, flop, shape):
        tf = flop / ms / 1e9
        res[name] = {"ms": ms, "tflops_algorithmic": tf, "frac_of_dgemm": tf / peak, "shape": shape}

    G, gam = rnd(n_nodes, n, n), rnd(n_nodes, n, n)
    w = torch.rand(n_nodes, dtype=torch.float64)
    products.gamma_sum(G, gam, 0, w)
    _, ms = _timed(torch, lambda: products.gamma_sum(G, gam, 0, w))
    rec("gamma_sum", ms, 8.0 * 2 * n_nodes * n ** 3, f"{n_nodes} nodes, G {n}x{n}, Gamma {n}x{n}")
    del G, gam

    g = rnd(n_bloch, 2 * n, 2 * n)
    hdl, sdl = rnd(n, n), rnd(n, n) * 0.05
    E = np.linspace(-1.0, 1.0, n_bloch)
    products.coupling_sigma(g, hdl, sdl, E)
    _, ms = _timed(torch, lambda: products.coupling_sigma(g, hdl, sdl, E))
    rec("bloch_coupling", ms, 8.0 * 2 * n_bloch * n ** 3, f"{n_bloch} energies, g {2 * n}x{2 * n}, H_DL {n}x{n}")
    del g

    ld = workload.random_device(n, 2, seed=seed).lead_L
    lead = LeadBlocks(ld.hL, ld.hLL, ld.sL, ld.sLL, ld.hDL, ld.sDL)
    El = np.linspace(-2.5, 2.5, n_lead_e)
    dec = self_energies(LeadArena([lead]), [0] * n_lead_e, El, eta, want_gs=True, check=False)
    gs = torch.stack(dec.gs)
    nc = ld.hDL.shape[0]
    gsig = rnd(n_lead_e, nc, nc)
    info = {}
    args = (ld.hL, ld.hLL, ld.sL, ld.sLL, ld.hDL, ld.sDL, El, eta, gs, gsig, 0)
    products.lead_adjoint(*args)
    _, ms = _timed(torch, lambda: products.lead_adjoint(*args, info=info))
    steps = info["iters"].astype(np.float64)
    # per energy: V and the explicit H_DL/S_DL terms (5 products), 4 products per doubling step, then
    # g tau', tau g tau', F^H Lambda, dW, dtau, tau g, dtau' (7 products) and one LU inverse (4/3 n^3)
    flop = 8.0 * n ** 3 * float(np.sum(5.0 + 7.0 + 4.0 / 3.0 + 4.0 * steps))
    rec("lead_adjoint", ms, flop, f"{n_lead_e} energies, lead {n}x{n}, H_DL {nc}x{ld.hDL.shape[1]}")
    res["lead_adjoint"]["doubling_steps_mean"] = float(steps.mean())
    res["note"] = ("each call timed once after a warm-up call, CUDA events around the Python API call; "
                   "work at 8 flop per complex multiply-add; frac against the in-run DGEMM")
    return res


def _ls_flops(n, iters):
    """Algorithmic FP64 work of one decimation: 8 (7/3 + 4) n^3 per doubling step (one solve with
    2n right-hand sides, four products) times the steps taken, plus 16 n^3 for g_s and Sigma."""
    return 8.0 * (7.0 / 3.0 + 4.0) * n ** 3 * iters + 16.0 * n ** 3


def _uneven_inputs(torch, n_devices, seed, first=0):
    """Devices first..first+n_devices-1 of the uneven set: b ~ U{16..256} (step 16) and
    L ~ U{8..64} drawn in device order from one seeded stream, their edge-block leads, and the
    energies: the far pole + 64 Ozaki poles at kT = 25 meV + 256 Gauss-Legendre points of the
    0.3 V bias window."""
    import numpy as np
    from dpnegf_b200 import rgf_plan, workload
    from dpnegf_b200.density import Ozaki
    from dpnegf_b200.scf import ozaki_weights
    from dpnegf_b200.surface_green import LeadBlocks
    rng = np.random.default_rng(seed)
    sizes = [(int(rng.integers(1, 17)) * 16, int(rng.integers(8, 65))) for _ in range(first + n_devices)]
    devs, leads, work = [], [], 0.0
    for d in range(first, first + n_devices):
        b, L = sizes[d]
        dev = workload.random_device(b, L, seed=seed + d)
        devs.append(rgf_plan.DeviceBlocks(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl))
        lb = lambda ld: LeadBlocks(ld.hL, ld.hLL, ld.sL, ld.sLL, ld.hDL, ld.sDL)
        leads.append((lb(dev.lead_L), lb(dev.lead_R)))
        work += 72.0 * b ** 3 * L
    kBT, mu_L, vL, vR = 0.025, 0.0, 0.15, -0.15
    oz = Ozaki(R=1e6, M_cut=64, n_gauss=256)
    fL = lambda x: 1.0 / (1.0 + torch.exp((x - (mu_L - vL)) / kBT))
    fR = lambda x: 1.0 / (1.0 + torch.exp((x - (mu_L - vR)) / kBT))
    z = ozaki_weights(oz.poles.numpy(), oz.residues.numpy(), oz.R, 256, kBT, mu_L, vL=vL, vR=vR, fermi_L=fL,
                      fermi_R=fR)[0]
    return dict(devs=devs, leads=leads, work=work, kBT=kBT, mu_L=mu_L, vL=vL, vR=vR, oz=oz, fL=fL, fR=fR, z=z)


def leads_leg(torch, peak, n_devices=128, seed=2024, eta=ETA_LEAD_SYNTH):
    """The uneven batch's decimation phase alone: both leads of every device at every energy in one
    Lopez-Sancho launch, timed with CUDA events, with its algorithmic FP64 rate against the
    measured DGEMM peak (per-item doubling steps from the kernel's own iteration counts)."""
    from dpnegf_b200.surface_green import LeadArena, self_energies
    u = _uneven_inputs(torch, n_devices, seed)
    nE = len(u["z"])
    arena = LeadArena([ld for pair in u["leads"] for ld in pair])
    idx = np.repeat(np.arange(2 * n_devices), nE)
    self_energies(arena, idx[:2 * nE], np.tile(u["z"], 2), eta, check=False)  # warm-up: module load
    res, ms = _timed(torch, lambda: self_energies(arena, idx, np.tile(u["z"], 2 * n_devices), eta, check=False))
    n = np.array([arena.shapes[i][0] for i in idx], dtype=np.float64)
    flops = float(_ls_flops(n, res.iters.astype(np.float64)).sum())
    ach = flops / (ms * 1e-3) / 1e12
    return {"items": int(len(idx)), "n": "16..256", "eta": eta, "seconds": ms * 1e-3,
            "value": len(idx) / (ms * 1e-3), "unit": "decimations/s", "mean_iters": float(res.iters.mean()),
            "max_iters": int(res.iters.max()), "status_counts": _status_counts(res.status),
            "roofline": {"achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
                         "algorithmic": "8 (7/3 + 4) n^3 per doubling step x steps + 16 n^3 per item"}}


def _status_counts(st):
    names = {0: "ok", 1: "warn_residual_1e-8", 2: "not_converged", 3: "residual_above_3e-5", 4: "singular"}
    v, c = np.unique(np.asarray(st), return_counts=True)
    return {names.get(int(a), str(int(a))): int(b) for a, b in zip(v, c)}


def metric_leads_leg(torch, peak, dev, E, eta=1e-5, n_energies=512):
    """Both leads of the metric device (its first / last block pairs repeated, b = 256) at
    ``n_energies`` energies of the grid, eta = 1e-5, one decimation launch: decimations/s, mean
    doubling steps and the algorithmic FP64 rate against the measured DGEMM peak."""
    from dpnegf_b200.surface_green import LeadArena, LeadBlocks, self_energies
    lb = lambda ld: LeadBlocks(ld.hL, ld.hLL, ld.sL, ld.sLL, ld.hDL, ld.sDL)
    arena = LeadArena([lb(dev.lead_L), lb(dev.lead_R)])
    Es = np.asarray(E.real.cpu().numpy())[cpu_sample_indices(len(E), n_energies)]
    idx = np.repeat([0, 1], len(Es))
    zz = np.tile(Es, 2)
    self_energies(arena, idx[:64], zz[:64], eta, check=False)  # warm-up
    res, ms = _timed(torch, lambda: self_energies(arena, idx, zz, eta, check=False))
    n = float(arena.shapes[0][0])
    flops = float(_ls_flops(n, res.iters.astype(np.float64)).sum())
    ach = flops / (ms * 1e-3) / 1e12
    return {"value": len(idx) / (ms * 1e-3), "unit": "decimations/s", "n": int(n), "items": int(len(idx)),
            "eta": eta, "iters_mean": float(res.iters.mean()), "seconds": ms * 1e-3,
            "status_counts": _status_counts(res.status),
            "roofline": {"achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
                         "algorithmic": "8 (7/3 + 4) n^3 per doubling step x steps + 16 n^3 per item "
                                        "(LU solve with 2n right-hand sides + 4 products per step)"},
            "workload": f"both edge-pair leads of the b=256 metric device, {len(Es)} energies of [-3, 3] eV"}


def uneven_leg(torch, n_devices=128, seed=2024, precisions=("fp64", "mixed", "mixed_refined"), chunk=128,
               eta_lead=ETA_LEAD_SYNTH):
    """The uneven batch (``_uneven_inputs``): every lead at every energy in one decimation launch,
    every (device, energy) item in one persistent sweep (Ozaki.uneven_batch), in chunks of
    ``chunk`` devices (the full batch's self-energies alone need about 100 GB), times summed.
    FP64, mixed, and mixed + FP64-residual refinement, the mixed runs checked against FP64; the
    decimation phase also timed alone."""
    from dpnegf_b200.surface_green import LeadArena, self_energies
    runs = (("fp64", "fp64", False), ("mixed", "mixed", False), ("mixed_refined", "mixed", True))
    ms = {tag: 0.0 for tag, _, _ in runs}
    ms_lead, work, items, nE, worst = 0.0, 0.0, 0, 0, {}
    timed = lambda fn: _timed(torch, fn)
    for first in range(0, n_devices, chunk):
        u = _uneven_inputs(torch, min(chunk, n_devices - first), seed, first=first)
        devs, leads, oz = u["devs"], u["leads"], u["oz"]
        kBT, mu_L, vL, vR, fL, fR, z = u["kBT"], u["mu_L"], u["vL"], u["vR"], u["fL"], u["fR"], u["z"]
        nd, nE = len(devs), len(z)
        arena = LeadArena([ld for pair in leads for ld in pair])
        ms_lead += timed(lambda: self_energies(arena, np.repeat(np.arange(2 * nd), nE), np.tile(z, 2 * nd),
                                               eta_lead))[1]
        del arena
        out = {}
        for tag, prec, refine in (r for r in runs if r[0] == "fp64" or r[0] in precisions):
            kw = dict(vL=vL, vR=vR, fermi_L=fL, fermi_R=fR, eta_lead=eta_lead, eta_device=1e-5, precision=prec,
                      refine=refine)
            out[tag], t = timed(lambda: oz.uneven_batch(devs, leads, kBT, mu_L, **kw))
            ms[tag] += t
        rel = lambda x, y: float((x - y).abs().max() / max(float(y.abs().max()), 1e-300))
        for tag in (t for t in ("mixed", "mixed_refined") if t in out):
            w = worst.setdefault(tag, [0.0, 0.0])
            w[0] = max(w[0], max(rel(m["n_eq"] + m["n_neq"], f["n_eq"] + f["n_neq"]) for m, f in zip(out[tag], out["fp64"])))
            w[1] = max(w[1], max(float((m["trans"] - f["trans"]).abs().max()) for m, f in zip(out[tag], out["fp64"])))
        work += u["work"] * nE
        items += nd * nE
        del out, devs, leads, u
        torch.cuda.empty_cache()
    res = {"devices": n_devices, "chunk": chunk, "energies_per_device": nE, "items": items,
           "eta_lead": eta_lead,
           "lead_decimation": {"items": 2 * items, "seconds": ms_lead * 1e-3},
           "fp64": {"value": items / (ms["fp64"] * 1e-3), "unit": "items/s", "seconds": ms["fp64"] * 1e-3,
                    "sweep_tflops_algorithmic": work / ((ms["fp64"] - ms_lead) * 1e-3) / 1e12}}
    for tag in worst:
        res[tag] = {"value": items / (ms[tag] * 1e-3), "unit": "items/s", "seconds": ms[tag] * 1e-3,
                    "density_rel_err_vs_fp64": worst[tag][0], "t_abs_err_vs_fp64": worst[tag][1]}
    return dict(res, **{
            "note": "per chunk: one call each (lead decimation + persistent sweep + density reduction), CUDA "
                    "events, summed over chunks; item = (device, energy); lead_decimation = that phase timed "
                    "alone; sweep_tflops counts 72 b^3 L per item over the FP64 time less the decimation's"})


def scf_leg(torch, peak, nk=8, n_energies=37, iters=10, eta_lead=ETA_LEAD_SYNTH):
    """b=512, L=40 at ``nk`` k-points (distinct H(k), S(k) realisations, equal weights): lead
    decimation on 512 x 512 blocks, then ``iters`` timed SCF iterations of damped (0.3) onsite
    shifts V = 0.5 (n - n0) around one sweep over every (k, energy) item, the iteration replayed as
    a CUDA graph (scf.ScfLoop).  Energies per k: the far pole + the Ozaki poles + bias-window
    points, ``n_energies`` in all (37 = 1 + 16 + 20 by default; 4096 = 1 + 64 + 4031 is the
    config's count).  FP64 and mixed; the mixed density checked against FP64."""
    import numpy as np
    from dpnegf_b200 import rgf_plan, workload
    from dpnegf_b200.ozaki_res_cal import ozaki_residues
    from dpnegf_b200.scf import ScfLoop, ozaki_weights
    from dpnegf_b200.surface_green import LeadArena, LeadBlocks, self_energies
    b, L = 512, 40
    devs = [workload.random_device(b, L, seed=512 + k) for k in range(nk)]
    kBT, mu_L, vL, vR = 0.025, 0.0, 0.15, -0.15
    n_poles = 16 if n_energies <= 37 else 64
    poles, res = ozaki_residues(n_poles)
    fL = lambda x: 1.0 / (1.0 + torch.exp((x - (mu_L - vL)) / kBT))
    fR = lambda x: 1.0 / (1.0 + torch.exp((x - (mu_L - vR)) / kBT))
    z, c, w = ozaki_weights(poles.numpy(), res.numpy(), 1e6, n_energies - 1 - n_poles, kBT, mu_L, vL=vL, vR=vR,
                            fermi_L=fL, fermi_R=fR)
    nE = len(z)
    lb = lambda ld: LeadBlocks(ld.hL, ld.hLL, ld.sL, ld.sLL, ld.hDL, ld.sDL)
    arena = LeadArena([lb(ld) for d in devs for ld in (d.lead_L, d.lead_R)])
    ls, t_lead = _timed(torch, lambda: self_energies(arena, np.repeat(np.arange(2 * nk), nE), np.tile(z, 2 * nk),
                                                     eta_lead))
    sig = [torch.stack(ls.sigma[i * nE:(i + 1) * nE]) for i in range(2 * nk)]
    del arena
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(d.hd, d.hu, d.hl, d.sd, d.su, d.sl) for d in devs])
    del devs
    out, ms = {}, {}
    for prec in ("fp64", "mixed"):
        loop = ScfLoop(geom, sig[0::2], sig[1::2], z, c, w, alpha=0.5, mix=0.3, eta=1e-5, precision=prec,
                       use_graph=True)
        loop.run(2)  # iteration 0 (sets n0) and iteration 1 (eager warm-up + graph capture), untimed
        (V, n), ms[prec] = _timed(torch, lambda: loop.run(2 + iters))
        out[prec] = (V.clone(), n.clone())
        loop.restore()
        del loop
    pts = nk * nE * iters  # one sweep over every (k, energy) item per replayed iteration
    ach = 72.0 * b ** 3 * L * pts / (ms["fp64"] * 1e-3) / 1e12
    rel = lambda x, y: float((x - y).abs().max() / max(float(y.abs().max()), 1e-300))
    return {"b": b, "L": L, "k_points": nk, "energies_per_k": nE, "iterations": iters,
            "lead_decimation": {"items": 2 * nk * nE, "seconds": t_lead * 1e-3, "n": b, "eta": eta_lead,
                                "status_counts": _status_counts(ls.status),
                                "mean_iters": float(ls.iters.mean()),
                                "tflops_algorithmic": float(_ls_flops(float(b), ls.iters.astype(np.float64)).sum())
                                / (t_lead * 1e-3) / 1e12},
            "fp64": {"value": pts / (ms["fp64"] * 1e-3), "unit": UNIT, "seconds": ms["fp64"] * 1e-3,
                     "roofline": {"achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak}},
            "mixed": {"value": pts / (ms["mixed"] * 1e-3), "unit": UNIT, "seconds": ms["mixed"] * 1e-3,
                      "speedup_vs_fp64": ms["fp64"] / ms["mixed"],
                      "n_rel_err_vs_fp64": rel(out["mixed"][1], out["fp64"][1]),
                      "V_rel_err_vs_fp64": rel(out["mixed"][0], out["fp64"][0])},
            "note": "energy points = k-points x energies x timed iterations; iterations 0-1 (equilibrium n0, "
                    "graph capture) untimed, then graph replays with the k-summed density reduction and the "
                    "potential update, CUDA events around them"}


def traffic_per_point(b, L):
    """DRAM bytes per energy point from the committed ncu summary, scaled by block count."""
    path = os.path.join(ROOT, "profiles", "rgf_kernel_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        if int(d["b"]) == b:
            return float(d["dram_bytes_per_point_per_block"]) * L
    except Exception:
        pass
    return None


def cpu_procs():
    """(processes, rule): one single-thread process per core, capped by 1.5 GB of free memory per
    process (each holds the b=256, L=64 device and its working blocks) and at 64."""
    n = os.cpu_count() or 1
    rule = f"min(os.cpu_count()={n}"
    try:
        import psutil
        mem_gb = psutil.virtual_memory().available / 2 ** 30
        n = min(n, max(1, int(mem_gb // 1.5)))
        rule += f", {mem_gb:.0f} GB available // 1.5 GB per process"
    except Exception:
        pass
    return max(1, min(n, 64)), rule + ", 64)"


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def workload_self_energies(B, b):
    """The self-energies every step of the GPU arm uses (seeds 1 and 2), on the host."""
    from dpnegf_b200 import workload
    return workload.random_self_energy(B, b, seed=1), workload.random_self_energy(B, b, seed=2)


def cpu_sample_indices(n_all, n_sample):
    return np.unique(np.linspace(0, n_all - 1, n_sample).round().astype(np.int64))


def cpu_baseline(args, seed, seL_h, seR_h, n_energies=0):
    """Oracle RGF + T/DOS on the host cores over a bounded sample of one step's workload: the
    device of k-seed ``seed`` at the sampled energies, with exactly the self-energies the GPU arm
    uses there, so the sample doubles as a parity check of that step (``T``/``D``/``idx``)."""
    from oracle import cpu_baseline as cb
    procs, rule = cpu_procs()
    nE = n_energies or args.cpu_energies or 8 * procs  # about 10-20 s of host work
    E_all = np.linspace(-3.0, 3.0, args.energies)
    idx = cpu_sample_indices(args.energies, nE)
    seL = seL_h[torch_index(idx)].numpy()
    seR = seR_h[torch_index(idx)].numpy()
    T, D, wall = cb.run_sample(args.b, args.L, seed, E_all[idx], seL, seR, args.eta, procs)
    return {"value": len(idx) / wall, "unit": UNIT, "cores": procs, "kind": "port", "seconds": wall,
            "energies": int(len(idx)), "cpu_model": cpu_model(), "cpu_count": os.cpu_count(),
            "process_rule": rule,
            "sample": f"{len(idx)} of the {args.energies} energies of the b={args.b} L={args.L} workload "
                      f"(k-seed {seed}, the GPU arm's self-energies at those energies), numpy oracle RGF + "
                      f"T/DOS, {procs} spawn processes x 1 BLAS thread, {wall:.1f} s",
            "T": T, "D": D, "idx": idx}


def torch_index(idx):
    import torch
    return torch.as_tensor(idx, dtype=torch.long)


def public_baseline(base):
    """The cpu_baseline object of the JSON line (without the sampled arrays)."""
    return {k: v for k, v in base.items() if k not in ("T", "D", "idx")}


def parity_vs_cpu(base, T_gpu, D_gpu):
    """Max relative differences of the GPU arm's T(E) and DOS from the CPU oracle at the sampled
    energies of the same device and self-energies."""
    idx = base["idx"]
    Tg, Dg = np.asarray(T_gpu)[idx], np.asarray(D_gpu)[idx]
    rel = lambda g, c: float(np.max(np.abs(g - c) / np.maximum(np.abs(c), 1e-300)))
    return {"t_max_rel_err": rel(Tg, base["T"]), "dos_max_rel_err": rel(Dg, base["D"]),
            "t_max_abs_err": float(np.max(np.abs(Tg - base["T"]))), "energies": int(len(idx)),
            "against": "oracle (numpy complex128 restatement of recursive_gf + _cal_tc_/_cal_dos_) on the "
                       "same device, energies and self-energies"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    seL_h, seR_h = workload_self_energies(args.energies, args.b)
    vals, secs = [], []
    base = None
    for s in range(args.warmup + args.steps):
        base = cpu_baseline(args, s, seL_h, seR_h)  # step s: the GPU arm's device of step s
        if s >= args.warmup:
            vals.append(base["value"])
            secs.append(base["seconds"])
    v = statistics.median(vals) if vals else base["value"]
    ms = 1e3 * (statistics.median(secs) if secs else base["seconds"])
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": f"random Hermitian TB device b={args.b} L={args.L}, energies in [-3,3] eV, "
                                   f"eta={args.eta}, T(E)+DOS; each step a bounded sample of "
                                   f"{base['energies']} energies on the host cores",
                       "b": args.b, "L": args.L, "energies_per_step": base["energies"]},
            "cpu_baseline": dict(public_baseline(base), value=v),
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

    # the CPU baseline pool is spawned before any CUDA work; it samples the first timed step
    # (device k-seed = warm-up count) with the GPU arm's own self-energies
    cpu_base = None
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    seL_h, seR_h = workload_self_energies(args.energies, args.b)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_base = cpu_baseline(args, args.warmup, seL_h, seR_h)

    import torch
    import torch.distributed as dist
    from dpnegf_b200 import _lib, rgf_plan, transport, workload

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    _lib.load()

    b, L, B = args.b, args.L, args.energies
    E = torch.linspace(-3.0, 3.0, B, dtype=torch.float64).to(torch.complex128)
    seL, seR = seL_h.cuda(), seR_h.cuda()
    Ed = E.cuda()
    nsteps = args.warmup + args.steps
    devs = [workload.random_device(b, L, seed=rank + world * s) for s in range(nsteps)]
    geoms = [rgf_plan.Geometry([rgf_plan.DeviceBlocks(d.hd, d.hu, d.hl, d.sd, d.su, d.sl)]) for d in devs]
    torch.cuda.synchronize()

    peak = measured_fp64_peak(torch)

    def barrier():
        if world > 1:
            dist.barrier()

    def step(s, ev=None, phase=False):
        return rgf_plan.run(geoms[s], [Ed], [seL], [seR], eta=args.eta, outputs=(), trans=True, dos=True,
                            check=False, events=ev, phase=phase, inverse=args.inverse)

    for s in range(args.warmup):
        r = step(s)
    torch.cuda.synchronize()
    st = r.status.cpu()
    assert int((st != 0).sum()) == 0, "warm-up produced failing items"

    clocks = Clocks(torch.cuda.current_device())
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    first = None
    for i in range(args.steps):
        r = step(args.warmup + i, ev=kev[i])
        if first is None:  # first timed step: its T/DOS are checked against the CPU sample
            first = r
    t1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = t0.elapsed_time(t1)
    kms = [a.elapsed_time(b_) for a, b_ in kev]
    if world > 1:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = world * B * args.steps / (ms * 1e-3)

    # roofline of the dominant kernel (rgf_kernel): algorithmic flops per launch / launch time
    k_avg = sum(kms) / len(kms)
    achieved = flops_per_point(b, L) * B / (k_avg * 1e-3) / 1e12
    tpp = traffic_per_point(b, L)
    roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": tpp * B if tpp else None, "kernel": "negf::rgf_kernel",
            "algorithmic": f"72*b^3*L flop/energy point (9 complex n^3 MACs per block, 4M count; "
                           f"3M products not credited) x {B} points per launch",
            "peak_source": "FP64 cuBLAS DGEMM 8192^3 measured in this run (of measured; "
                           "MEASURED_PEAKS.json has no FP64 figure)"}

    phases = None
    if args.phases:
        phases = {}
        for prec in ("fp64", "mixed"):
            r = rgf_plan.run(geoms[args.warmup], [Ed], [seL], [seR], eta=args.eta, outputs=(), trans=True,
                             dos=True, check=False, phase=True, precision=prec, inverse=args.inverse)
            torch.cuda.synchronize()
            pc = r.phase_cycles.sum(0).double()
            phases[prec] = {n: float(v) for n, v in zip(_lib.PHASES, (pc / pc.sum()).tolist()) if v > 0}

    # mixed precision and adjoint legs (rank 0): same devices, 1 warm-up + 1 timed step each
    mixed = adjoint = None
    T64 = None  # FP64 kernel T(E) of the first timed device (error reference of the other legs)
    if rank == 0 and not args.no_mixed:
        sref = args.warmup  # first timed device; its FP64 T/DOS are the error reference
        r64 = step(sref)
        torch.cuda.synchronize()
        T64, D64 = r64.trans.cpu(), r64.dos.cpu()

        def leg(fn):
            fn(0)
            torch.cuda.synchronize()
            a, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            out = fn(sref)
            b_.record()
            torch.cuda.synchronize()
            return out, a.elapsed_time(b_)

        def mstep(s, **kw):
            return rgf_plan.run(geoms[s], [Ed], [seL], [seR], eta=args.eta, outputs=(), trans=True, dos=True,
                                check=False, precision="mixed", **kw)

        rm, msm = leg(lambda s: mstep(s))
        rr, msr = leg(lambda s: mstep(s, refine=True, refine_steps=args.refine_steps))
        tf32 = measured_tf32_peak(torch)
        v_m, v_r = B / (msm * 1e-3), B / (msr * 1e-3)
        ach_m = flops_per_point(b, L) * v_m / 1e12
        mixed = {
            "value": v_m, "unit": UNIT, "speedup_vs_fp64": v_m / value,
            "t_abs_err_max": float((rm.trans.cpu() - T64).abs().max()),
            "dos_rel_err_max": float(((rm.dos.cpu() - D64).abs() / D64.abs()).max()),
            "refined": {"value": v_r, "unit": UNIT, "speedup_vs_fp64": v_r / value,
                        "refine_steps_max": args.refine_steps,
                        "t_abs_err_max": float((rr.trans.cpu() - T64).abs().max())},
            "roofline": {"bound": "tensor", "achieved": ach_m, "peak": tf32, "unit": "TFLOP/s",
                         "frac": ach_m / tf32,
                         "tensor_frac_executed": 3.0 * ach_m / tf32,
                         "peak_source": "cuBLAS TF32 GEMM 8192^3 measured in this run (of measured)",
                         "note": "algorithmic 72*b^3*L flop per point as for FP64; the 3xTF32 split "
                                 "executes 3x that on the tensor cores"},
            "precision": "complex products as 3xTF32 split on tcgen05.mma kind::tf32 (FP32 accumulation "
                         "in TMEM); pivoting, panels and storage FP64; refined = FP64-residual steps on "
                         "G_{:,N} (early stop at 1e-10 relative)",
            "timing": f"1 warm-up + 1 timed step ({B} energies), CUDA events, rank 0"}
        w = torch.ones(B, dtype=torch.float64)
        adjoint = {}
        for prec in ("fp64", "mixed"):
            def fwd(s, prec=prec):
                return rgf_plan.run(geoms[s], [Ed], [seL], [seR], eta=args.eta, outputs=(), trans=True,
                                    check=False, precision=prec)

            def adj(s, prec=prec):
                return rgf_plan.run(geoms[s], [Ed], [seL], [seR], eta=args.eta, outputs=(), check=False,
                                    adjoint_w=w, precision=prec)
            _, tf = leg(fwd)
            _, ta = leg(adj)
            adjoint[prec] = {"value": B / ((tf + ta) * 1e-3), "unit": UNIT,
                             "forward_value": B / (tf * 1e-3), "grad_over_forward": ta / tf,
                             "fused_value": B / (ta * 1e-3)}
        adjoint["mixed_vs_fp64"] = adjoint["mixed"]["value"] / adjoint["fp64"]["value"]
        adjoint["current_density_b96_L32"] = current_density_leg(torch, rgf_plan, workload, args.eta)
        adjoint["note"] = ("value = energy points/s of T(E) plus the full gradient d(sum T)/d(all H, S "
                           "blocks, both self-energies) through autograd (forward launch + adjoint launch); "
                           "fused_value = the same T(E) and gradient from the single adjoint launch "
                           "(adjoint.transmission_and_grad, for weights known in advance); grad_over_forward = "
                           "adjoint launch time / T-only forward time; 1 warm-up + 1 timed step each")

    # the reference's own GPU path (torch complex128 solve + matmul) on a sample of the same workload
    # lead self-energies of the metric device at eta = 1e-5 (rank 0)
    leads = None
    if rank == 0 and not args.no_leads and devs[args.warmup].lead_L is not None:
        leads = metric_leads_leg(torch, peak, devs[args.warmup], E)

    torch_ref = None
    if rank == 0 and args.torch_energies > 0:
        d = devs[args.warmup]
        Tt, idx, tms = torch_reference_leg(torch, d, E, seL, seR, args.eta, args.torch_energies)
        if T64 is None:
            r64 = step(args.warmup)
            torch.cuda.synchronize()
            T64 = r64.trans.cpu()
        terr = float((Tt.cpu() - T64[idx]).abs().max())
        torch_ref = {"value": args.torch_energies / (tms * 1e-3), "unit": UNIT, "kind": "port",
                     "speedup_of_fp64_kernel": value / (args.torch_energies / (tms * 1e-3)),
                     "t_abs_err_vs_fp64_kernel": terr,
                     "sample": f"{args.torch_energies} of the {B} energies (same device, self-energies), "
                               f"batches of 32, 1 warm-up pass + best of 2 timed passes, CUDA events",
                     "path": "torch complex128 restatement of recursive_gf's stacked GPU branch "
                             "(torch.linalg.solve + batched matmul on cuSOLVER/cuBLAS) and "
                             "DeviceProperty._cal_tc_/_cal_dos_, on this B200"}
        if mixed:
            torch_ref["mixed_adjoint_speedup"] = adjoint["mixed"]["value"] / torch_ref["value"]
            torch_ref["mixed_adjoint_fused_speedup"] = adjoint["mixed"]["fused_value"] / torch_ref["value"]
            torch_ref["fp64_adjoint_fused_speedup"] = adjoint["fp64"]["fused_value"] / torch_ref["value"]
            torch_ref["mixed_speedup"] = mixed["value"] / torch_ref["value"]
            torch_ref["mixed_refined_speedup"] = mixed["refined"]["value"] / torch_ref["value"]

    extra = {}
    if rank == 0 and args.configs:
        wanted = [x.strip() for x in args.configs.split(",") if x.strip()]
        if "leads" in wanted:
            extra["config3_leads"] = leads_leg(torch, peak, n_devices=args.lead_devices, eta=args.lead_eta)
        if "uneven" in wanted:
            extra["config3_uneven"] = uneven_leg(torch, n_devices=args.uneven_devices,
                                                 precisions=args.uneven_precisions.split(","),
                                                 chunk=args.uneven_chunk, eta_lead=args.lead_eta)
        if "scf" in wanted:
            extra["config5_scf"] = scf_leg(torch, peak, nk=args.scf_k, n_energies=args.scf_energies,
                                           iters=args.scf_iters, eta_lead=args.lead_eta)
    # the product chains (default line, or asked for with --configs products)
    if rank == 0 and (not args.no_products or "products" in args.configs.split(",")):
        extra["product_chains"] = products_leg(torch, peak, eta=args.lead_eta)

    # end-to-end through the public API: pinned host inputs, host outputs
    e2e = None
    if not args.no_e2e:
        d = devs[args.warmup]
        pin = lambda xs: [x.contiguous().pin_memory() for x in xs]
        hd, hu, hl, sd, su, sl = pin(d.hd), pin(d.hu), pin(d.hl), pin(d.sd), pin(d.su), pin(d.sl)
        Eh, sLh, sRh = E.pin_memory(), seL_h.pin_memory(), seR_h.pin_memory()
        h2d = sum(x.numel() * 16 for x in hd + hu + hl + sd + su + sl) + (sLh.numel() + sRh.numel() + Eh.numel()) * 16
        d2h = 2 * B * 8
        transport.transmission_dos(hd, hu, hl, sd, su, sl, Eh, sLh, sRh, eta=args.eta)  # warm
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        n_e2e = 1
        for _ in range(n_e2e):
            T, D, _ = transport.transmission_dos(hd, hu, hl, sd, su, sl, Eh, sLh, sRh, eta=args.eta)
        e1.record()
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        if world > 1:
            tt = torch.tensor([ems], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ems = float(tt.item())
        e2e = {"value": world * B * n_e2e / (ems * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h,
               "path": "dpnegf_b200.transport.transmission_dos with pinned host H/S blocks, self-energies "
                       "and energies; T(E) and DOS returned to host"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
                "path": "fp64",
                "config": {"workload": f"random Hermitian TB device b={b} L={L}, {B} energies in [-3,3] eV per "
                                       f"k-realisation (step), eta={args.eta}, complex128, T(E)+DOS fused",
                           "b": b, "L": L, "energies_per_step": B, "k_per_step_per_gpu": 1,
                           "l2": "inputs larger than L2 (H/S arena 380 MiB per step, per-slot scratch 82 MiB x 148)",
                           "parallelism": f"k-realisations across {world} GPU(s)"},
                "roofline": roof, "cpu_baseline": public_baseline(cpu_base) if cpu_base else None,
                "parity": parity_vs_cpu(cpu_base, first.trans.cpu().numpy(), first.dos.cpu().numpy())
                if cpu_base else None, "e2e": e2e, "clocks": clk,
                "gpu_launches": args.steps, "kernel_ms": kms}
        if phases:
            line["phases"] = phases
        if mixed:
            line["mixed"] = mixed
            line["adjoint"] = adjoint
        if torch_ref:
            line["torch_gpu_reference"] = torch_ref
        if leads:
            line["leads"] = leads
        line.update(extra)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
