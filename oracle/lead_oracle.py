"""numpy restatement of the reference lead self-energy and density helpers.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Citations are relative
to the dpnegf source tree.
"""
import numpy as np

# status codes shared with the CUDA path (include/negf_b200.h)
LS_OK, LS_WARN, LS_NOT_CONVERGED, LS_RESIDUAL = 0, 1, 2, 3


def surface_green(H, h01, S, s01, ee, max_iter=100, tol=1e-40):
    """Lopez-Sancho decimation; returns ``(gs, status, iterations, residual)``.

    Follows ``_surface_green_numba_core`` (negf/surface_green.py:102-159):
    alpha = h10 - ee s10, beta = h01 - ee s01, eps = epss = H; each iteration
    solves (ee S - eps) [Xa Xb] = [alpha beta] and updates
    eps += alpha Xb + beta Xa, epss += beta Xa, alpha <- alpha Xa,
    beta <- beta Xb; converged when max(|alpha| + |beta|) < 1e-40; then
    gs = (ee S - epss)^-1 and the residual max|(ee S - H - (ee s01 - h01) gs
    (ee s10 - h10)) gs - I| must be < 3e-5 (warn above 1e-8).  The reference
    raises ArithmeticError / RuntimeError where this returns a status.
    """
    H = np.asarray(H, np.complex128)
    h01 = np.asarray(h01, np.complex128)
    S = np.asarray(S, np.complex128)
    s01 = np.asarray(s01, np.complex128)
    ee = complex(ee)
    n = H.shape[0]
    h10 = h01.conj().T
    s10 = s01.conj().T
    alpha = h10 - ee * s10
    beta = h01 - ee * s01
    eps = H.copy()
    epss = H.copy()
    eS = ee * S
    for it in range(1, max_iter + 2):
        sol = np.linalg.solve(eS - eps, np.concatenate([alpha, beta], axis=1))
        xa, xb = sol[:, :n], sol[:, n:]
        b_xa = beta @ xa
        eps = eps + alpha @ xb + b_xa
        epss = epss + b_xa
        alpha = alpha @ xa
        beta = beta @ xb
        if np.max(np.abs(alpha) + np.abs(beta)) < tol:
            gs = np.linalg.inv(eS - epss)
            test = eS - H - (ee * s01 - h01) @ gs @ (ee * s10 - h10)
            res = np.max(np.abs(test @ gs - np.eye(n)))
            if res < 3.0e-5:
                return gs, (LS_WARN if res > 1.0e-8 else LS_OK), it, res
            return gs, LS_RESIDUAL, it, res
        if it >= max_iter + 1:
            break
    return None, LS_NOT_CONVERGED, max_iter + 1, np.inf


def self_energy(hL, hLL, sL, sLL, ee, hDL=None, sDL=None, etaLead=1e-8, E_ref=0.0):
    """Sigma = (E sDL - hDL) gs[:b,:b] (E sDL^H - hDL^H)  (negf/surface_green.py:9-91).

    ``E = ee + E_ref`` and the decimation runs at ``E + 1j*etaLead``
    (:65-70, :83).  Without ``hDL`` the bulk form ``ESH - gs^-1`` (:73-80)
    is returned.  Returns ``(Sigma, gs, status, iterations)``.
    """
    E = complex(ee) + complex(E_ref)
    gs, st, it, _ = surface_green(hL, hLL, sL, sLL, E + 1j * etaLead)
    if gs is None:
        return None, None, st, it
    if hDL is None:
        sig = (E * np.asarray(sL) - np.asarray(hL)) - np.linalg.inv(gs)
    else:
        hDL = np.asarray(hDL, np.complex128)
        sDL = np.asarray(sDL, np.complex128)
        b = hDL.shape[1]
        sig = (E * sDL - hDL) @ gs[:b, :b] @ (E * sDL.conj().T - hDL.conj().T)
    return sig, gs, st, it


def ozaki_residues(M_cut):
    """Poles and residues of the Ozaki continued fraction (negf/ozaki_res_cal.py:8-37).

    The 2M x 2M tridiagonal matrix has zero diagonal and off-diagonal
    1/(2 sqrt((2n-1)(2n+1))), n = 1..2M-1; its positive eigenvalues lam give
    poles 1/lam (ascending) and residues |v_0|^2 / (4 lam^2).
    """
    from scipy.linalg import eigh_tridiagonal
    N = 2 * int(M_cut)
    off = np.array([0.5 / np.sqrt((2.0 * n - 1) * (2.0 * n + 1)) for n in range(1, N)])
    ev, evec = eigh_tridiagonal(np.zeros(N), off, select="i", select_range=(N // 2, N - 1))
    return np.flip(1.0 / ev).copy(), np.flip(np.abs(evec[0, :]) ** 2 / (4.0 * ev ** 2)).copy()


def gauss_xw(xl, xu, n):
    """Gauss-Legendre nodes/weights mapped to [xl, xu] (negf/negf_utils.py:136-160)."""
    x, w = np.polynomial.legendre.leggauss(n)
    return x * (0.5 * (xu - xl)) + 0.5 * (xu + xl), w * 0.5 * (xu - xl)


def gauss_xw_f32(xl, xu, n):
    """``gauss_xw`` as ``Ozaki.integrate`` evaluates it (negf/density.py:186, negf_utils.py:153-158):
    the limits come from ``torch.scalar_tensor`` (float32), so nodes and weights are float32."""
    x, w = np.polynomial.legendre.leggauss(n)
    xl32, xu32 = np.float32(xl), np.float32(xu)
    half = np.float32(0.5) * (xu32 - xl32)
    return x.astype(np.float32) * half + np.float32(0.5) * (xu32 + xl32), w.astype(np.float32) * half


def ozaki_density(gf, mu_L, mu_D, kBT, R, M_cut, n_gauss, vL, vR, fermi_L, fermi_R, gamma_R_fn):
    """Restatement of ``Ozaki.integrate`` (negf/density.py:143-199) with explicit mu.

    The reference reads ``deviceprop.mu`` and ``deviceprop.lead_L.mu``, which
    its classes never define; here they are the arguments ``mu_D`` and
    ``mu_L``.  ``gf(z)`` must return the device Green block G(z) used by the
    reference (``grd[0]``) and ``gamma_R_fn(e)`` the right-lead Gamma at real
    energy ``e`` (embedded to the size of ``grd[0]``).

    DM_eq = Re[ iR G(iR - mu_D) - sum_p Im(-4 i kT G(z_p) r_p) ],
    z_p = i pole_p kT + mu_L - mu_D;
    DM_neq = sum_i w_i Re[G Gamma_R G^H] (f_R - f_L) at Gauss-Legendre points
    on [min(vL,vR) - 8kT, max(vL,vR) + 8kT] when the bias is non-zero; nodes, weights, the Fermi
    factors at x + mu_D and their difference are float32 there, as the reference forms them
    (``fermi_L`` / ``fermi_R`` receive a float32 argument).
    """
    poles, res = ozaki_residues(M_cut)
    zp = 1j * poles * kBT + mu_L - mu_D
    dm = 1j * R * gf(1j * R - mu_D)
    for i, z in enumerate(zp):
        dm = dm - np.imag((-4j * kBT) * gf(z) * res[i])
    dm_eq = np.real(dm)
    if abs(vL - vR) > 1e-14:
        xl, xu = min(vL, vR) - 8 * kBT, max(vL, vR) + 8 * kBT
        xs, wl = gauss_xw_f32(xl, xu, n_gauss)
        dm_neq = 0.0
        for x, w in zip(xs, wl):
            G = gf(complex(x))
            a = np.real(G @ gamma_R_fn(complex(x)) @ G.conj().T)
            e = x + np.float32(mu_D)
            df = np.float32(fermi_R(e)) - np.float32(fermi_L(e))
            dm_neq = dm_neq + w * (a * df)
    else:
        dm_neq = 0.0
    return dm_eq, dm_neq


def current_nscf(energy_grid, tc, efermi, kBT):
    """I-V sweep by Simpson integration (negf/device_property.py:333-371)."""
    from scipy.integrate import simpson
    f = lambda x, mu: 1.0 / (1.0 + np.exp((x - mu) / kBT))
    emin, emax = energy_grid.min(), energy_grid.max()
    vmin, vmax = emin + 4 * kBT, emax - 4 * kBT
    vm = 0.5 * (vmin + vmax)
    vmid = vm - vmin
    # the bias grid is float32 there (torch.linspace in the default dtype); each half-bias dv enters
    # the float64 chemical potentials with its float32 value
    vv = np.linspace(0.0, vmid, int(vmid / 0.1) + 1).astype(np.float32) * np.float32(2)
    cc = [simpson(y=(f(energy_grid + efermi, efermi - vm + float(dv)) - f(energy_grid + efermi, efermi - vm - float(dv)))
                  * tc, x=energy_grid) for dv in vv * np.float32(0.5)]
    return vv, np.array(cc)


def fiori_subblock_index(subblocks, atom_index, norbs):
    """Blocks holding an atom's orbitals, with the start offset in the first of them and the end
    offset in the last (negf/density.py:362-395): scan the block edges for the block holding the
    first orbital, then extend block by block until the last orbital is covered."""
    edges = [0]
    for n in subblocks:
        edges.append(edges[-1] + int(n))
    first = int(sum(norbs[:atom_index]))
    last = first + int(norbs[atom_index])
    for i in range(len(edges) - 1):
        if edges[i] <= first and last <= edges[i + 1]:
            return [i], first - edges[i], last - edges[i]
        if edges[i] <= first < edges[i + 1] < last:
            blocks = [i]
            for j in range(i + 1, len(edges) - 1):
                blocks.append(j)
                if last <= edges[j + 1]:
                    return blocks, first - edges[i], last - edges[j]
    raise ValueError(f"atom {atom_index} lies outside the blocks")


def fiori_free_charge(energies, pre_factor, blocks, left_se, right_se, eta_device, E_ref_device, fermi_L, fermi_R,
                      E_ref, norbs, potential_at_atom, block_tridiagonal, subblocks):
    """Restatement of ``Fiori.density_integrate_Fiori`` (negf/density.py:268-360), one energy at a time.

    ``blocks`` = (hd, hu, hl, sd, su, sl); ``left_se`` / ``right_se`` hold one self-energy per
    energy.  For each energy: A_R = G Gamma_R G^H from the full block (dense device) or from the
    last block column G_qN (BTD device), A_L = i(G_qq - G_qq^H) - A_R, G^n = A_L f_L + A_R f_R,
    G^p = A_L + A_R - G^n, f at E + E_ref; then per atom  w (-1/pi) Tr G^n  if E >= -potential
    (electrons) else  w (1/pi) Tr G^p  (holes), the trace taken over the atom's orbitals block by
    block as the reference slices them.  Returns the complex [n_atoms] charge."""
    from . import rgf_oracle
    hd, hu, hl, sd, su, sl = blocks
    charge = np.zeros(len(norbs), dtype=np.complex128)
    edges = np.concatenate([[0], np.cumsum(norbs)])
    for i, e in enumerate(energies):
        out = rgf_oracle.rgf(complex(e), hl, hd, hu, sd, su, sl, left_se[i], right_se[i], E_ref=E_ref_device,
                             eta=eta_device, need_gr_lc=True)
        grd = [x[0] for x in out["grd"]]
        gam = rgf_oracle.gamma_from_se(np.asarray(right_se[i]))
        ty = grd[-1].shape[-1]
        x1 = min(gam.shape[0], ty)
        if not block_tridiagonal:
            GR = np.zeros((ty, ty), dtype=np.complex128)
            GR[ty - x1:, ty - x1:] = gam[gam.shape[0] - x1:, gam.shape[1] - x1:]
            A_R = [grd[0] @ GR @ grd[0].conj().T]
        else:
            gR = gam[gam.shape[0] - x1:, gam.shape[1] - x1:]
            A_R = [c[0] @ gR @ c[0].conj().T for c in out["gr_lc"]]
        A_L = [1j * (g - g.conj().T) - a for g, a in zip(grd, A_R)]
        fl, fr = fermi_L(e + E_ref), fermi_R(e + E_ref)
        gn = [al * fl + ar * fr for al, ar in zip(A_L, A_R)]
        gp = [al + ar - n for al, ar, n in zip(A_L, A_R, gn)]
        for a, Ei in enumerate(-1 * np.asarray(potential_at_atom)):
            electron = e >= Ei
            M = gn if electron else gp
            coef = pre_factor[i] * 2 * (-1) / 2 / np.pi if electron else pre_factor[i] * 2 * 1 / 2 / np.pi
            if not block_tridiagonal:
                tr = np.trace(M[0][edges[a]:edges[a + 1], edges[a]:edges[a + 1]])
            else:
                bl, s0, s1 = fiori_subblock_index(subblocks, a, norbs)
                if len(bl) == 1:
                    tr = np.trace(M[bl[0]][s0:s1, s0:s1])
                else:
                    tr = np.trace(M[bl[0]][s0:, s0:]) + np.trace(M[bl[-1]][:s1, :s1])
                    tr = tr + sum(np.trace(M[b]) for b in bl[1:-1])
            charge[a] += coef * tr
    return charge
