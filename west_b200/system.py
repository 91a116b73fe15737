"""Synthetic Gamma-point plane-wave systems: the implicit inputs of Wstat's
response operator.

``apply_operator`` (Wstat/apply_operator.f90:14) reads its ground state from
Quantum ESPRESSO module variables: ``evc``, ``et``, ``g2kin``, ``vrs``,
``vkb``, ``deeq``, ``dffts%nl/nlm``, ``omega``, ``wk`` and the Coulomb factor
``pot3D%sqvc``.  This module builds those arrays for an orthorhombic (by
default cubic) cell filled with Gaussian pseudo-atoms, in QE's conventions:

* Rydberg units; kinetic energy ``g2kin = |G|^2 tpiba2``; ``e2 = 2``.
* Gamma-only storage: the half sphere ``x > 0 | (x = 0, y > 0) | (x = y = 0,
  z >= 0)`` with ``psi(-G) = conj(psi(G))``, sorted by ``|G|^2`` so that G=0
  comes first (``gstart = 2`` in Fortran numbering).
* ``nl``/``nlm``: box positions of +G / -G in an ``nr1 x nr2 x nr3`` box, x fastest.
  They are returned 0-based here; the C ABI takes QE's 1-based values.
* ``invfft`` is the unscaled sum over ``exp(+iGr)``; ``fwfft`` carries 1/N^3.

The ground state comes from an exact diagonalisation of the same Hamiltonian
the response operator applies (kinetic + local potential sampled on the FFT
box + Kleinman-Bylander projectors), written as a real symmetric matrix on
the Gamma half sphere.  With no aliasing in the box (2*Gmax < nr/2) the dense
matrix equals the FFT-based ``h_psi`` exactly.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

E2 = 2.0          # e^2 in Rydberg units (QE constants: e2)
FPI = 4.0 * math.pi


@dataclasses.dataclass(frozen=True)
class SystemSpec:
    """Parameters of a synthetic orthorhombic (default cubic) Gamma-only system."""
    L: float | tuple         # cell edge (bohr), or (Lx, Ly, Lz)
    ecutwfc: float           # wavefunction cutoff (Ry)
    nr: int | tuple          # FFT box edge, or (nr1, nr2, nr3)
    natoms: int              # Gaussian pseudo-atoms at seeded uniform positions
    nbnd_occ: int            # occupied bands
    proj: str = "s"          # "s" or "sp": KB projectors per atom
    Z: float = 4.0           # local well depth (Ry): V(r) = -Z exp(-r^2 / 2 sigma^2)
    sigma: float = 0.8       # local well width (bohr)
    sigma_p: float = 0.6     # Gaussian radial width of the KB projectors (bohr)
    dion: float = 1.0        # KB coupling D (Ry), diagonal
    nbnd_extra: int = 4      # empty bands computed beside the occupied ones
    seed: int = 0
    frac_occ: tuple = ()     # occupations of the highest occupied bands (fractional
                             # occupations, QE's wg / wk); the others are 1


def cell_lengths(L) -> tuple:
    """(Lx, Ly, Lz) of a cell given as one edge or three."""
    return tuple(float(x) for x in L) if isinstance(L, (tuple, list)) else (float(L),) * 3


def box_edges(nr) -> tuple:
    """(nr1, nr2, nr3) of a box given as one edge or three."""
    return tuple(int(x) for x in nr) if isinstance(nr, (tuple, list)) else (int(nr),) * 3


# Workloads.  c1..c5 follow the five named configurations; ``tiny``/``small``
# are the sizes the CPU tests run in seconds.
SPECS = {
    "tiny": SystemSpec(L=8.0, ecutwfc=6.0, nr=16, natoms=2, nbnd_occ=3, proj="sp", seed=11),
    "small": SystemSpec(L=10.0, ecutwfc=8.0, nr=24, natoms=3, nbnd_occ=7, proj="sp", seed=12),
    "c1": SystemSpec(L=15.0, ecutwfc=20.0, nr=48, natoms=4, nbnd_occ=8, proj="s", seed=1),
    "c2": SystemSpec(L=20.0, ecutwfc=25.0, nr=64, natoms=8, nbnd_occ=32, proj="sp", seed=2),
    "c4a": SystemSpec(L=15.0, ecutwfc=20.0, nr=48, natoms=4, nbnd_occ=8, proj="sp", seed=41),
    "c4b": SystemSpec(L=20.0, ecutwfc=25.0, nr=64, natoms=8, nbnd_occ=32, proj="sp", seed=42),
    "c4c": SystemSpec(L=25.0, ecutwfc=25.0, nr=80, natoms=12, nbnd_occ=64, proj="sp", seed=43),
    "c5": SystemSpec(L=30.0, ecutwfc=30.0, nr=108, natoms=20, nbnd_occ=128, proj="sp", seed=5),
}


@dataclasses.dataclass
class GammaSystem:
    """All arrays the response operator consumes (QE/WEST naming)."""
    spec: SystemSpec
    omega: float
    tpiba2: float
    nr: int | tuple         # box edge (cubic) or (nr1, nr2, nr3)
    mill: np.ndarray        # int32 [npw, 3] Miller indices, |G| order, G=0 first
    g2kin: np.ndarray       # f64 [npw]
    nl: np.ndarray          # int64 [npw] 0-based box index of +G
    nlm: np.ndarray         # int64 [npw] 0-based box index of -G
    vrs: np.ndarray         # f64 [nr1 nr2 nr3] local potential on the box (x fastest)
    vkb: np.ndarray         # c128 [npw, nkb]
    deeq: np.ndarray        # f64 [nkb, nkb]
    evc: np.ndarray         # c128 [npw, nbnd_occ]
    et: np.ndarray          # f64 [nbnd_occ + nbnd_extra]
    occupation: np.ndarray  # f64 [nbnd_occ]
    sqvc: np.ndarray        # f64 [npw]
    alpha_pv: float
    wk: float = 2.0         # QE k weight at Gamma, non-spin-polarised (sum = 2)
    tau: Optional[np.ndarray] = None

    @property
    def npw(self) -> int:
        return int(self.mill.shape[0])

    @property
    def nbnd_occ(self) -> int:
        return int(self.evc.shape[1])

    @property
    def nkb(self) -> int:
        return int(self.vkb.shape[1])

    @property
    def nrs(self) -> tuple:
        return box_edges(self.nr)

    @property
    def nnr(self) -> int:
        n1, n2, n3 = self.nrs
        return n1 * n2 * n3


def gamma_half_sphere(L, ecutwfc: float, nr):
    """Miller indices of the Gamma half sphere |G|^2 <= ecutwfc (Ry, bohr^-2) of an
    orthorhombic cell L (one edge or three) in the box nr (one edge or three),
    sorted by |G|^2 (ties by Miller index) so that G=0 is first.  Returns
    (mill, tpiba2) with tpiba2 = (2 pi / Lx)^2 (QE's alat = Lx)."""
    Ls, ns = cell_lengths(L), box_edges(nr)
    b = [2.0 * math.pi / x for x in Ls]
    nmax = [int(math.sqrt(ecutwfc) / bi) + 1 for bi in b]
    i, j, k = np.meshgrid(np.arange(-nmax[0], nmax[0] + 1), np.arange(-nmax[1], nmax[1] + 1),
                          np.arange(-nmax[2], nmax[2] + 1), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    if Ls[0] == Ls[1] == Ls[2]:        # cubic: integer |m|^2 as the sort key, exact ties
        key = i * i + j * j + k * k
        g2 = key * b[0] ** 2
    else:
        g2 = (i * b[0]) ** 2 + (j * b[1]) ** 2 + (k * b[2]) ** 2
        key = g2
    keep = (g2 <= ecutwfc) & ((i > 0) | ((i == 0) & (j > 0)) | ((i == 0) & (j == 0) & (k >= 0)))
    mill = np.stack([i[keep], j[keep], k[keep]], axis=1).astype(np.int32)
    order = np.lexsort((mill[:, 2], mill[:, 1], mill[:, 0], key[keep]))
    mill = mill[order]
    for d in range(3):
        if np.abs(mill[:, d]).max() * 2 >= ns[d]:
            raise ValueError(f"FFT box {ns} too small for cutoff {ecutwfc} Ry in cell {Ls}")
    return mill, b[0] ** 2


def g2_of(mill: np.ndarray, L) -> np.ndarray:
    """|G|^2 (bohr^-2 = Ry) of Miller triples in the orthorhombic cell L."""
    b = np.array([2.0 * math.pi / x for x in cell_lengths(L)])
    return ((mill.astype(np.float64) * b[None, :]) ** 2).sum(1)


def box_index(mill: np.ndarray, nr) -> np.ndarray:
    """0-based linear index (x fastest) of Miller triples in the box nr."""
    n1, n2, n3 = box_edges(nr)
    m = mill.astype(np.int64)
    return np.mod(m[:, 0], n1) + n1 * (np.mod(m[:, 1], n2) + n2 * np.mod(m[:, 2], n3))


def _local_potential(L, nr, tau, Z, sigma):
    (Lx, Ly, Lz), (n1, n2, n3) = cell_lengths(L), box_edges(nr)
    x = np.arange(n1) * (Lx / n1)
    y = np.arange(n2) * (Ly / n2)
    z = np.arange(n3) * (Lz / n3)
    v = np.zeros((n3, n2, n1))          # [k][j][i] = (z, y, x)
    for t in tau:
        dx = x - t[0]; dx -= Lx * np.round(dx / Lx)
        dy = y - t[1]; dy -= Ly * np.round(dy / Ly)
        dz = z - t[2]; dz -= Lz * np.round(dz / Lz)
        d2 = dz[:, None, None] ** 2 + dy[None, :, None] ** 2 + dx[None, None, :] ** 2
        v += -Z * np.exp(-d2 / (2.0 * sigma * sigma))
    return v.ravel()


def _kb_projectors(mill, L, tau, proj, sigma_p):
    b = np.array([2.0 * math.pi / x for x in cell_lengths(L)])
    G = mill.astype(np.float64) * b[None, :]               # [npw, 3] bohr^-1
    g2 = (G * G).sum(1)
    radial = np.exp(-0.5 * sigma_p * sigma_p * g2)
    cols = []
    for t in tau:
        phase = np.exp(-1j * (G @ np.asarray(t)))
        cols.append(radial * phase)                        # s
        if proj == "sp":
            for a in range(3):                             # p_x, p_y, p_z (real in r space)
                cols.append(-1j * sigma_p * G[:, a] * radial * phase)
    vkb = np.stack(cols, axis=1)
    # unit norm under the Gamma dot product 2 sum_half |b|^2 - |b(0)|^2
    nrm = 2.0 * (np.abs(vkb) ** 2).sum(0) - np.abs(vkb[0]) ** 2
    return vkb / np.sqrt(nrm)[None, :]


def _dense_gamma_hamiltonian(sysd, device="cpu"):
    """Real symmetric Hamiltonian on the orthonormal Gamma basis
    {e_0, (e_G + e_-G)/sqrt2, i(e_G - e_-G)/sqrt2}."""
    import torch
    n1, n2, n3 = box_edges(sysd["nr"])
    mill = torch.as_tensor(sysd["mill"].astype(np.int64), device=device)
    vt = np.fft.fftn(sysd["vrs"].reshape(n3, n2, n1)) / (n1 * n2 * n3)   # V(G) on the box
    vt = torch.as_tensor(vt.ravel(), device=device)
    npw = mill.shape[0]
    nn = torch.as_tensor([n1, n2, n3], device=device)

    def vidx(sign):
        d = (mill[:, None, :] + sign * mill[None, :, :]) % nn
        return d[..., 0] + n1 * (d[..., 1] + n2 * d[..., 2])

    B = torch.as_tensor(sysd["vkb"], device=device)
    D = torch.as_tensor(sysd["deeq"], device=device).to(B.dtype)
    hpp = vt[vidx(-1)]                       # H(G, G')
    hpp += B @ D @ B.conj().T
    hpp += torch.diag(torch.as_tensor(sysd["g2kin"], device=device)).to(hpp.dtype)
    hpq = vt[vidx(+1)]                       # H(G, -G')
    hpq += B @ D @ B.T
    H = torch.empty((2 * npw, 2 * npw), dtype=torch.float64, device=device)
    H[:npw, :npw] = hpp.real + hpq.real
    H[npw:, npw:] = hpp.real - hpq.real
    H[:npw, npw:] = -hpp.imag + hpq.imag
    H[npw:, :npw] = H[:npw, npw:].T
    del hpp, hpq
    # G = 0 has no sine partner; its cosine vector is sqrt2 * e_0
    s = 1.0 / math.sqrt(2.0)
    H[0, :] *= s
    H[:, 0] *= s
    keep = torch.ones(2 * npw, dtype=torch.bool, device=device)
    keep[npw] = False
    return H[keep][:, keep]


# Real Gamma basis dimension above which the lowest bands come from the
# iterative solver (the dense eigensolver needs (2 npw)^2 doubles and its
# 64-bit cuSOLVER path rejects n > 32768).
DENSE_MAX_DIM = 20000


def _fix_signs(evc):
    # only a sign is free (psi(r) stays real): make the largest real part positive
    for b in range(evc.shape[1]):
        k = np.argmax(np.abs(evc[:, b].real))
        if evc[k, b].real < 0:
            evc[:, b] *= -1.0
    return evc


def _ground_state(sysd, nbnd, device="cpu"):
    import torch
    npw = sysd["mill"].shape[0]
    if 2 * npw - 1 > DENSE_MAX_DIM:
        return _ground_state_iterative(sysd, nbnd, device=device)
    H = _dense_gamma_hamiltonian(sysd, device=device)
    H = 0.5 * (H + H.T)
    w, v = torch.linalg.eigh(H)
    w = w[:nbnd].cpu().numpy()
    x = v[:, :nbnd].cpu().numpy()
    evc = np.empty((npw, nbnd), dtype=np.complex128)
    evc[0] = x[0]
    s = 1.0 / math.sqrt(2.0)
    evc[1:] = (x[1:npw] + 1j * x[npw:]) * s
    return w, _fix_signs(evc)


class _GammaH:
    """Matrix-free H on the Gamma half sphere (psi(-G) = conj psi(G)): kinetic,
    local potential through the FFT box (QE invfft unscaled, fwfft with 1/N^3)
    and Kleinman-Bylander projectors with the Gamma bra-ket 2 Re sum - G0."""

    def __init__(self, sysd, device):
        import torch
        nr = sysd["nr"]
        mill = sysd["mill"]
        self.nrs = box_edges(nr)
        n1, n2, n3 = self.nrs
        self.nl = torch.as_tensor(box_index(mill, nr), device=device)
        self.nlm = torch.as_tensor(box_index(-mill, nr), device=device)
        self.v = torch.as_tensor(sysd["vrs"].reshape(n3, n2, n1), device=device)
        self.g2 = torch.as_tensor(sysd["g2kin"], device=device)
        self.B = torch.as_tensor(sysd["vkb"], device=device)
        self.D = torch.as_tensor(sysd["deeq"], device=device).to(self.B.dtype)
        self.chunk = max(1, int(2e9 // (16 * n1 * n2 * n3)))   # vectors per FFT batch (about 2 GB of boxes)

    def dot(self, a, b):
        """Gamma Gram matrix <a_i|b_j> (real)."""
        import torch
        return 2.0 * (a.conj().T @ b).real - torch.outer(a[0].conj(), b[0]).real

    def __call__(self, psi):
        import torch
        n1, n2, n3 = self.nrs
        out = torch.empty_like(psi)
        for c0 in range(0, psi.shape[1], self.chunk):
            p = psi[:, c0:c0 + self.chunk]
            k = p.shape[1]
            box = torch.zeros((k, n1 * n2 * n3), dtype=torch.complex128, device=psi.device)
            box[:, self.nlm] = p.T.conj()
            box[:, self.nl] = p.T                       # G = 0: the +G store wins (psi(0) is real)
            r = torch.fft.ifftn(box.view(k, n3, n2, n1), dim=(1, 2, 3), norm="forward") * self.v
            g = torch.fft.fftn(r, dim=(1, 2, 3), norm="forward").reshape(k, -1)
            out[:, c0:c0 + k] = g[:, self.nl].T
        out += self.g2[:, None] * psi
        becp = self.dot(self.B, psi)
        out += self.B @ (self.D @ becp.to(self.B.dtype))
        out[0].imag.zero_()                             # Im hpsi(G = 0) = 0
        return out


def _ground_state_iterative(sysd, nbnd, device="cpu", tol=1e-9, maxit=500, seed=7):
    """Lowest nbnd eigenpairs by block LOBPCG on the Gamma half sphere: Rayleigh-Ritz
    over [X, T R, P] orthonormalised in the Gamma metric, T = 1 / (1 + g2kin) the
    kinetic preconditioner, stopped when every wanted residual is below tol."""
    import torch
    H = _GammaH(sysd, device)
    npw = sysd["mill"].shape[0]
    k = nbnd + max(4, nbnd // 8)                        # guard vectors
    gen = torch.Generator().manual_seed(seed)
    X = torch.complex(torch.randn(npw, k, generator=gen, dtype=torch.float64),
                      torch.randn(npw, k, generator=gen, dtype=torch.float64)).to(device)
    X = X / (1.0 + H.g2[:, None])
    X[0].imag.zero_()
    prec = 1.0 / (1.0 + H.g2)

    def ortho(Y):
        S = H.dot(Y, Y)
        w, U = torch.linalg.eigh(0.5 * (S + S.T))
        keep = w > w.max() * 1e-13
        return Y @ (U[:, keep] / torch.sqrt(w[keep])).to(Y.dtype)

    X = ortho(X)
    HX = H(X)
    P = None
    th = None
    for _ in range(maxit):
        A = H.dot(X, HX)
        th, C = torch.linalg.eigh(0.5 * (A + A.T))
        C = C.to(X.dtype)
        X, HX = X @ C, HX @ C
        R = HX - X * th[None, :].to(X.dtype)
        rn = torch.sqrt(torch.clamp(torch.diagonal(H.dot(R, R)), min=0.0))
        if float(rn[:nbnd].max()) < tol:
            break
        W = R * prec[:, None]
        W[0].imag.zero_()
        Q = ortho(torch.cat([X, W] + ([P] if P is not None else []), 1))
        HQ = H(Q)
        A = H.dot(Q, HQ)
        _, C = torch.linalg.eigh(0.5 * (A + A.T))
        C = C[:, :k].to(Q.dtype)
        Xn = Q @ C
        P = Xn - X @ H.dot(X, Xn).to(X.dtype)
        X, HX = Xn, HQ @ C
    w = th[:nbnd].cpu().numpy()
    evc = X[:, :nbnd].cpu().numpy().astype(np.complex128)
    evc[0] = evc[0].real
    return w, _fix_signs(evc)


def build_system(spec: SystemSpec | str, device: Optional[str] = None) -> GammaSystem:
    """Build a synthetic Gamma system from a spec (or the name of one)."""
    if isinstance(spec, str):
        spec = SPECS[spec]
    if device is None:
        device = "cpu"
    rng = np.random.default_rng(spec.seed)
    L, nr = spec.L, spec.nr
    Ls = cell_lengths(L)
    mill, tpiba2 = gamma_half_sphere(L, spec.ecutwfc, nr)
    tau = rng.uniform(0.0, 1.0, size=(spec.natoms, 3)) * np.array(Ls)[None, :]
    if Ls[0] == Ls[1] == Ls[2]:
        g2kin = (mill.astype(np.float64) ** 2).sum(1) * tpiba2
    else:
        g2kin = g2_of(mill, L)
    nl = box_index(mill, nr)
    nlm = box_index(-mill, nr)
    vrs = _local_potential(L, nr, tau, spec.Z, spec.sigma)
    vkb = _kb_projectors(mill, L, tau, spec.proj, spec.sigma_p)
    nkb = vkb.shape[1]
    deeq = np.eye(nkb) * spec.dion
    sysd = dict(nr=nr, mill=mill, vrs=vrs, vkb=vkb, deeq=deeq, g2kin=g2kin)
    nbnd = spec.nbnd_occ + spec.nbnd_extra
    et, evc = _ground_state(sysd, nbnd, device=device)
    qg2 = g2kin.copy()
    sqvc = np.zeros_like(qg2)
    nz = qg2 > 1e-8
    sqvc[nz] = np.sqrt(E2 * FPI / qg2[nz])           # Coulomb_kernel/class_coulomb.f90:173
    emin = et.min()
    emax = et[: spec.nbnd_occ].max()
    alpha_pv = max(2.0 * (emax - emin), 0.01)          # Tools/get_alpha_pv.f90:59-63
    occ = np.ones(spec.nbnd_occ)
    if spec.frac_occ:
        occ[spec.nbnd_occ - len(spec.frac_occ):] = np.asarray(spec.frac_occ, dtype=np.float64)
    return GammaSystem(
        spec=spec, omega=Ls[0] * Ls[1] * Ls[2], tpiba2=tpiba2, nr=nr, mill=mill, g2kin=g2kin,
        nl=nl, nlm=nlm, vrs=vrs, vkb=vkb, deeq=deeq,
        evc=np.ascontiguousarray(evc[:, : spec.nbnd_occ]), et=et,
        occupation=occ, sqvc=sqvc, alpha_pv=alpha_pv, tau=tau)


def perturbations(sysm: GammaSystem, m: int, seed: int = 1234) -> np.ndarray:
    """dvg test batch: seeded complex-normal coefficients times 4 pi / |G|^2
    (G = 0 zeroed), column-major [npw, m]."""
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((sysm.npw, m)) + 1j * rng.standard_normal((sysm.npw, m))
    scale = np.zeros(sysm.npw)
    nz = sysm.g2kin > 1e-8
    scale[nz] = FPI / sysm.g2kin[nz]
    return np.asfortranarray(z * scale[:, None])


def randomized_basis(sysm: GammaSystem, m: int, seed: int = 4321) -> np.ndarray:
    """Starting PDEP guesses in the manner of do_randomize
    (Wstat/davidson_diago.f90:1121-1182): amplitude rr uniform in [0,1), phase
    2 pi uniform, divided by (|g|^2 + 1) with g in 2pi/alat units; G=0 left 0."""
    rng = np.random.default_rng(seed)
    rr = rng.random((sysm.npw, m))
    arg = 2.0 * math.pi * rng.random((sysm.npw, m))
    g2 = sysm.g2kin / sysm.tpiba2
    a = rr * np.exp(1j * arg) / (g2 + 1.0)[:, None]
    a[0] = 0.0
    return np.asfortranarray(a)
