"""CPU oracle of the vertical remap (test infrastructure only): the
incompressible remap_vertical_coordinates of src/remap.f90, restated with
numpy over every node column of one level at once.

  remap_incompressible  src/remap.f90:147-216 (porosity 1)
  find_coordinates_incompressible  :235-257 (z_new = a_vert eta + b_vert z_s)
  remap0    :259-285   piecewise constant
  remap1    :287-380   piecewise linear, harmonic-mean slopes, ENHANCE (10 rounds)
  remap2PPM :382-495   PPM with limited slopes, Dirichlet ends

Every expression keeps the reference's operand order, so the CUDA kernel
(csrc/remap_kernels.cuh, FP64 without FMA contraction) matches it bit for bit.
Columns are the second axis: var[k, c] with k = 1..N at rows 1..N (row 0
unused), z[k, c] with k = 0..N."""
import numpy as np

from .grid import own


def remap0(N, z_new, v_old, z_old):
    FC = np.zeros_like(z_old)
    for k in range(1, N):
        dz = z_new[k] - z_old[k]
        FC[k] = np.minimum(dz, 0.0) * v_old[k] + np.maximum(dz, 0.0) * v_old[k + 1]
    v_new = np.zeros_like(v_old)
    for k in range(1, N + 1):
        v_new[k] = ((z_old[k] - z_old[k - 1]) * v_old[k] + FC[k] - FC[k - 1]) / (z_new[k] - z_new[k - 1])
    return v_new


def remap1(N, z_new, v_old, z_old):
    Hz = np.zeros_like(z_old)
    FC = np.zeros_like(z_old)
    aL = np.zeros_like(z_old)
    aR = np.zeros_like(z_old)
    for k in range(1, N + 1):
        Hz[k] = z_old[k] - z_old[k - 1]
    for k in range(N - 1, 0, -1):
        FC[k] = (v_old[k + 1] - v_old[k]) / (Hz[k + 1] + Hz[k])
    FC[0] = FC[1]
    FC[N] = FC[N - 1]
    with np.errstate(all="ignore"):
        for k in range(1, N + 1):
            cff = np.where(FC[k] * FC[k - 1] < 0.0, 0.0, 2 * FC[k] * FC[k - 1] / (FC[k] + FC[k - 1]))
            aR[k] = v_old[k] + cff * Hz[k]
            aL[k] = v_old[k] - cff * Hz[k]
    for _ in range(10):
        for k in range(1, N):
            FC[k] = 0.5 * (aR[k] + aL[k + 1])
        FC[N] = aR[N]
        FC[0] = aL[1]
        for k in range(1, N + 1):
            dR = FC[k] - v_old[k]
            dL = v_old[k] - FC[k - 1]
            cff = np.where(dR * dL < 0.0, 0.0, np.where(np.abs(dR) > np.abs(dL), dL, dR))
            aR[k] = v_old[k] + cff
            aL[k] = v_old[k] - cff
    for k in range(1, N):
        dz = z_new[k] - z_old[k]
        up = dz > 0.0
        cff = np.where(up, aL[k + 1], aR[k])
        cff1 = np.where(up, aR[k + 1] - aL[k + 1], aR[k] - aL[k])
        dh = np.where(up, Hz[k + 1], Hz[k])
        FC[k] = dz * (cff + 0.5 * cff1 * dz / dh)
    FC[0] = 0.0
    FC[N] = 0.0
    v_new = np.zeros_like(v_old)
    for k in range(1, N + 1):
        v_new[k] = (Hz[k] * v_old[k] + FC[k] - FC[k - 1]) / (z_new[k] - z_new[k - 1])
    return v_new


def remap2ppm(N, z_new, v_old, z_old):
    Hz, aL, aR, CF, FC, FC1 = (np.zeros_like(z_old) for _ in range(6))
    for k in range(1, N + 1):
        Hz[k] = z_old[k] - z_old[k - 1]
    for k in range(1, N):
        cff = 1.0 / (Hz[k] + Hz[k + 1])
        CF[k] = cff * (v_old[k + 1] * Hz[k] + v_old[k] * Hz[k + 1])
        FC[k] = cff * (v_old[k + 1] - v_old[k])
    for k in range(2, N):
        cff = Hz[k] * ((2.0 * Hz[k - 1] + Hz[k]) * FC[k] + (2.0 * Hz[k + 1] + Hz[k]) * FC[k - 1]) / \
            (Hz[k - 1] + Hz[k] + Hz[k + 1])
        cffR = 2.0 * (v_old[k + 1] - v_old[k])
        cffL = 2.0 * (v_old[k] - v_old[k - 1])
        same = cffR * cffL > 0.0
        c1 = np.where(np.abs(cffL) < np.abs(cff), cffL, cff)
        c2 = np.where(np.abs(cffR) < np.abs(c1), cffR, c1)
        FC1[k] = np.where(same, c2, 0.0)
    FC1[N] = Hz[N] * FC[N - 1]
    FC1[1] = Hz[1] * FC[1]
    for k in range(1, N):
        k1, k2 = max(k - 1, 1), min(k + 2, N)
        cff = Hz[k1] + Hz[k] + Hz[k + 1] + Hz[k2]
        cffL = (Hz[k1] + Hz[k]) / (cff * (2.0 * Hz[k] + Hz[k + 1]))
        cffR = (Hz[k + 1] + Hz[k2]) / (cff * (Hz[k] + 2.0 * Hz[k + 1]))
        aR[k] = CF[k] + 2.0 * Hz[k] * Hz[k + 1] * (cffL - cffR) * FC[k] - cffL * Hz[k] * FC1[k + 1] + \
            cffR * Hz[k + 1] * FC1[k]
        aL[k + 1] = aR[k]
    aR[N] = 2.0 * v_old[N] - aL[N]
    aL[1] = 2.0 * v_old[1] - aR[1]
    for k in range(1, N + 1):
        CF[k] = 0.5 * (aR[k] - aL[k])
        FC[k] = 0.5 * (aR[k] + aL[k]) - v_old[k]
    for k in range(1, N):
        dz = z_new[k] - z_old[k]
        up = dz > 0.0
        alpha = np.where(up, Hz[k + 1], -Hz[k])
        cff = np.where(up, aL[k + 1], aR[k])
        cffR = np.where(up, CF[k + 1], -CF[k])
        cffL = np.where(up, FC[k + 1], FC[k])
        alpha = dz / alpha
        FC[k] = dz * (cff + alpha * (cffR - cffL * (3.0 - 2.0 * alpha)))
    FC[0] = 0.0
    FC[N] = 0.0
    v_new = np.zeros_like(v_old)
    for k in range(1, N + 1):
        v_new[k] = (Hz[k] * v_old[k] + FC[k] - FC[k - 1]) / (z_new[k] - z_new[k - 1])
    return v_new


REMAP = {"0": remap0, "1": remap1, "2PPM": remap2ppm}


def coordinates(topo, mean_m, mass_old, a_vert, b_vert, rho0):
    """find_coordinates_incompressible for every slot: (z_new, z_old), (N+1, NN)."""
    nz = mass_old.shape[0]
    zo = np.zeros((nz + 1, topo.size))
    zo[0] = topo
    for k in range(1, nz + 1):
        rho_dz = mean_m[k - 1] + mass_old[k - 1]
        zo[k] = zo[k - 1] + rho_dz / (rho0 * 1.0)
    eta = zo[nz]
    zn = np.stack([a_vert[k] * eta + b_vert[k] * topo for k in range(nz + 1)])
    return zn, zo


def remap_level(lv, nz, state, remap_type, a_vert, b_vert, rho0):
    """remap_incompressible on every own-source node of [0, n]^2 of one level
    (pole slots: masses and Theta only).  state: mass, temp, velo, mean_m,
    mean_t, topo as in the C-ABI layout.  Returns new (mass, temp, velo);
    other slots keep their values."""
    lv = own(lv)
    n, P, NN = lv.n, lv.P, lv.NN
    nsrc = np.arange(NN)
    nsrc[lv.halo_node[:, 0]] = lv.halo_node[:, 1]
    mass, temp, velo = (np.array(state[k], dtype=np.float64).copy() for k in ("mass", "temp", "velo"))
    mm, mt, topo = state["mean_m"], state["mean_t"], np.asarray(state["topo"], dtype=np.float64)
    zn_all, zo_all = coordinates(topo[nsrc], mm[:, nsrc], mass[:, nsrc], a_vert, b_vert, rho0)
    d, j, i = np.meshgrid(np.arange(10), np.arange(n + 1), np.arange(n + 1), indexing="ij")
    x = ((d * P + j + 2) * P + i + 2).ravel()
    ii, jj = i.ravel(), j.ravel()
    keep = nsrc[x] == x
    x, ii, jj = x[keep], ii[keep], jj[keep]
    pole = (ii == n) | (jj == n)
    f = REMAP[remap_type]
    pad = np.zeros((1, x.size))
    zn, zo = zn_all[:, x], zo_all[:, x]
    dz = zn[1:] - zn[:-1]
    # edge velocities, columns averaged with the node at each edge's far end
    xv = x[~pole]
    for e, off in enumerate((1, P + 1, P)):
        xr = nsrc[xv + off]
        zen = 0.5 * (zn_all[:, xv] + zn_all[:, xr])
        zeo = 0.5 * (zo_all[:, xv] + zo_all[:, xr])
        vo = np.vstack([pad[:, :xv.size], velo[:, e * NN + xv]])
        vn = f(nz, zen, vo, zeo)
        velo[:, e * NN + xv] = vn[1:]
    theta = np.vstack([pad, (mt[:, x] + temp[:, x]) / (mm[:, x] + mass[:, x])])
    tn = f(nz, zn, theta, zo)
    rho_dz = (rho0 * 1.0) * dz
    mass[:, x] = rho_dz - mm[:, x]
    temp[:, x] = rho_dz * tn[1:] - mt[:, x]
    return mass, temp, velo


def min_mass_level(lv, nz, state, b_vert, rho0, mask_n=None):
    """cal_min_mass (src/main.f90:642-693), incompressible case, A/B hybrid
    grid, porosity 1, over the own-source nodes of [0, n]^2 of one level whose
    node mask is at least ADJZONE (8; every node without masks): the smallest
    (sol + sol_mean) / (rho0 dz_k) with dz_k = b_vert[k+1] z_s - b_vert[k] z_s.
    A layer mass that is not positive, or a ratio that is not, gives 0 (where
    the reference aborts); no node gives 1e16, the reference's start value."""
    lv = own(lv)
    n, P, NN = lv.n, lv.P, lv.NN
    nsrc = np.arange(NN)
    nsrc[lv.halo_node[:, 0]] = lv.halo_node[:, 1]
    d, j, i = np.meshgrid(np.arange(10), np.arange(n + 1), np.arange(n + 1), indexing="ij")
    x = ((d * P + j + 2) * P + i + 2).ravel()
    x = x[nsrc[x] == x]
    if mask_n is not None:
        x = x[np.asarray(mask_n)[x] >= 8]
    if x.size == 0:
        return 1e16
    b = np.asarray(b_vert, dtype=np.float64)
    zs = np.asarray(state["topo"], dtype=np.float64)[x]
    rho_dz = np.asarray(state["mass"])[:, x] + np.asarray(state["mean_m"])[:, x]
    dz = b[1:, None] * zs[None, :] - b[:-1, None] * zs[None, :]
    with np.errstate(all="ignore"):
        rel = rho_dz / (rho0 * dz)
    if not ((rho_dz > 0.0) & (rel > 0.0)).all():
        return 0.0
    return float(rel.min())
