"""Self-consistent onsite potential with the sweep replayed as a CUDA graph.

One iteration of the loop:

  H_qq(k) <- H0_qq(k) + diag(V_q)                  (every k-point, in the packed H/S arena)
  sweep over every (k, energy) item                 (one persistent launch)
  n_i    = sum_k wk [Re sum_e c_e diag(G_k(z_e))_i + sum_e w_e diag(G_qN Gamma_R G_qN^H)_k(x_e)_i]
  V      <- V + mix * (alpha * (n - n0) - V)        (damped onsite shifts)

with n0 the equilibrium density of the unshifted device, so the charge
that the bias window moves drives the potential.  The weights come from
``ozaki_weights``: c = iR at the far pole and 4 kT r_p at the Ozaki poles
(the equilibrium density of negf/density.py:164-181 written as one weighted
sum), w = w_GL (f_R - f_L) on the bias-window Gauss-Legendre points
(:183-195).  The leads do not depend on V, so their self-energies are
computed once.  Iteration 0 runs eagerly (it sets n0 and checks the item
status); the iteration body is then captured once in a CUDA graph and
replayed, so an SCF step costs one graph launch and no host work.  After k
iterations ``n`` is the density of the potential before the k-th update and
``V`` carries k updates.
"""
from typing import Optional

import numpy as np
import torch
import torch.distributed as dist

from . import rgf_plan
from .negf_utils import gauss_xw


def ozaki_weights(poles, residues, R, n_gauss, kBT, mu_L, mu_D=0.0, vL=0.0, vR=0.0, fermi_L=None,
                  fermi_R=None):
    """Energies (relative to E_ref) and density weights of the Ozaki + bias-window quadrature.

    Returns ``(z, c, w)``: complex energies [B], complex weights of diag(G(z))
    [B] and real weights of the spectral diagonal [B] (zero on the poles)."""
    poles = np.asarray(poles, dtype=np.float64)
    res = np.asarray(residues, dtype=np.float64)
    z = np.concatenate([[1j * R - mu_D], 1j * poles * kBT + mu_L - mu_D]).astype(np.complex128)
    c = np.concatenate([[1j * R], 4.0 * kBT * res]).astype(np.complex128)
    w = np.zeros(len(z))
    if abs(vL - vR) > 1e-14:
        xl, xu = min(vL, vR) - 8 * kBT, max(vL, vR) + 8 * kBT
        xs, wl = gauss_xw(xl=torch.scalar_tensor(xl, dtype=torch.float64),
                          xu=torch.scalar_tensor(xu, dtype=torch.float64), n=n_gauss)
        df = (fermi_R(xs + mu_D) - fermi_L(xs + mu_D)).real
        z = np.concatenate([z, xs.numpy().astype(np.complex128)])
        c = np.concatenate([c, np.zeros(len(xs), dtype=np.complex128)])
        w = np.concatenate([w, (wl * df).numpy()])
    return z, c, w


class ScfLoop:
    """Damped onsite-potential SCF of a BTD device around a captured sweep.

    ``geometry`` holds the device at one or more k-points (one
    ``DeviceBlocks`` per k, the same orbitals in each); ``se_left`` /
    ``se_right`` are the lead self-energies at every energy of ``z``
    ([B, n, n], e.g. from ``surface_green.self_energies``), or one such stack
    per k-point.  The density is the ``wk``-weighted sum of the k-point
    densities (equal weights by default), as the runner sums k contributions
    (runner/NEGF.py:904-906), and the one potential shifts every k-point's
    onsite blocks; every (k, energy) item runs in the same launch.  ``z, c, w``
    from ``ozaki_weights``.  ``alpha`` is the onsite response (eV per
    electron) and ``mix`` the damping.  ``precision`` selects the FP64 or the
    mixed sweep.

    Over several ranks (``group``, or the default process group when one is
    initialised with more than one rank) each rank passes its own k-points and
    their weights; the k-summed density is all-reduced once per iteration
    (one vector of n_orb values), outside the captured graph, and every rank
    then applies the same potential update.  ``plan``: a deferred plan for
    ``geometry`` at ``z`` with per-orbital outputs (``rgf_plan.run(...,
    orb_g=True, orb_ar=bias, defer=True)``), built here when omitted.
    """

    def __init__(self, geometry: rgf_plan.Geometry, se_left, se_right, z, c, w, alpha=0.5, mix=0.3, eta=0.0,
                 E_ref=0.0, precision="fp64", use_graph=True, wk=None, group=None, plan=None):
        nk = len(geometry.devs)
        if not isinstance(se_left, (list, tuple)):
            se_left, se_right = [se_left], [se_right]
        if len(se_left) != nk or len(se_right) != nk:
            raise ValueError(f"one left and one right self-energy stack per k-point ({nk})")
        if len({int(d["n_orb"]) for d in geometry.devs}) != 1:
            raise ValueError("every k-point must carry the same orbitals")
        wk = np.full(nk, 1.0 / nk) if wk is None else np.asarray(wk, dtype=np.float64).reshape(-1)
        if len(wk) != nk:
            raise ValueError(f"{len(wk)} k weights for {nk} k-points")
        self.geom = geometry
        dev = geometry.device
        idx = []
        for d in geometry.devs:
            for q in range(int(d["blk0"]), int(d["blk0"]) + int(d["n_blocks"])):
                b = geometry.blocks[q]
                n = int(b["n"])
                idx.append(int(b["hd"]) + np.arange(n) * (n + 1))
        self.diag_idx = torch.as_tensor(np.concatenate(idx), device=dev)
        self.h0 = geometry.hs[self.diag_idx].clone()
        self.nk = nk
        self.n_orb = int(geometry.devs[0]["n_orb"])
        self.B = len(z)
        self.wk = torch.as_tensor(wk, dtype=torch.float64, device=dev).reshape(nk, 1)
        self.c = torch.as_tensor(np.asarray(c), dtype=torch.complex128, device=dev).reshape(-1, 1)
        self.w = torch.as_tensor(np.asarray(w), dtype=torch.float64, device=dev).reshape(-1, 1)
        self.bias = bool(np.any(np.asarray(w) != 0))
        self.alpha, self.mix = float(alpha), float(mix)
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
        if plan is None:
            E = torch.as_tensor(np.asarray(z), dtype=torch.complex128, device=dev)
            plan = rgf_plan.run(geometry, [E] * nk, list(se_left), list(se_right), eta=eta, E_ref=E_ref,
                                outputs=(), orb_g=True, orb_ar=self.bias, precision=precision, defer=True)
        self.plan = plan
        self.V = torch.zeros(self.n_orb, dtype=torch.float64, device=dev)
        self.n = torch.zeros(self.n_orb, dtype=torch.float64, device=dev)
        self.n0: Optional[torch.Tensor] = None
        self.use_graph = use_graph
        self.graph = None
        self.iterations = 0

    def _density(self, equilibrium_only=False):
        r = self.plan.result
        n = (self.c * r.orb_g.view(self.nk, self.B, self.n_orb)).real.sum(1)
        if self.bias and not equilibrium_only:
            n = n + (self.w * r.orb_ar.view(self.nk, self.B, self.n_orb)).sum(1)
        return (self.wk * n).sum(0)

    def _update(self):
        self.V.add_(self.mix * (self.alpha * (self.n - self.n0) - self.V))

    def _sum_ranks(self, x):
        if self.world > 1:
            dist.all_reduce(x, op=dist.ReduceOp.SUM, group=self.group)
        return x

    def _body(self):
        """Shift, sweep and this rank's density; the update too when one rank holds every k-point
        (then the whole iteration is one graph)."""
        self.geom.hs.index_copy_(0, self.diag_idx, self.h0 + self.V.to(torch.complex128).repeat(self.nk))
        self.plan.launch()
        self.n.copy_(self._density())
        if self.world == 1:
            self._update()

    def _finish(self):
        """Over several ranks: the density summed over every rank's k-points, then the update."""
        if self.world > 1:
            self._sum_ranks(self.n)
            self._update()

    def step(self):
        """One SCF iteration; returns the density of that iteration's potential."""
        if self.n0 is None:  # iteration 0: unshifted device, eager, sets n0
            self.geom.hs.index_copy_(0, self.diag_idx, self.h0 + self.V.to(torch.complex128).repeat(self.nk))
            self.plan.launch()
            self.plan.check()
            self.n0 = self._sum_ranks(self._density(equilibrium_only=True).clone())
            self.n.copy_(self._sum_ranks(self._density()))
            self._update()
            self.iterations = 1
            return self.n
        if self.use_graph and self.graph is None:
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                self._body()  # eager warm-up of the body on a side stream (also iteration 1)
            torch.cuda.current_stream().wait_stream(s)
            self._finish()
            self.plan.check()
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph, capture_error_mode="relaxed"):
                self._body()
            self.iterations += 1
            return self.n
        if self.graph is not None:
            self.graph.replay()
        else:
            self._body()
        self._finish()
        self.iterations += 1
        return self.n

    def run(self, iterations=10):
        for _ in range(iterations - self.iterations):
            self.step()
        if self.geom.device.type == "cuda":
            torch.cuda.current_stream().synchronize()
        self.plan.check()
        return self.V, self.n

    def restore(self):
        """Put the unshifted onsite blocks back into the arena."""
        self.geom.hs.index_copy_(0, self.diag_idx, self.h0)
