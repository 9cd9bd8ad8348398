"""Seeded synthetic periodic systems for the short-range nonbonded path.

The reference measures on no public dataset; these generators build the
water / water+solute boxes its workloads describe, in the units and encodings
SPONGE's modules receive:

* coordinates in Angstrom as float32 ``VECTOR`` triples, unwrapped;
* charges pre-multiplied by SPONGE's internal charge scale 18.2223
  (``SPONGE/common.h`` ``CONSTANT_SPONGE_CHARGE_SCALE``), so q_i*q_j/r is in
  kcal/mol;
* LJ pair tables in SPONGE's internal convention: ``A = 12*4*eps*sigma^12``,
  ``B = 6*4*eps*sigma^6`` (the native loader multiplies the file's A by 12 and
  B by 6, ``SPONGE/xponge/load/native/lj.hpp:47,57``), stored in the
  triangular order ``idx(a,b) = max*(max+1)/2 + min``
  (``SPONGE/Lennard_Jones_force/Lennard_Jones_force.h:18-27``);
* exclusions as the upper-triangular CSR triple (``excluded_list_start``,
  ``excluded_numbers``, ``excluded_list``) that ``MD_core/nb.hpp:30-70``
  builds;
* the lower-triangular cell ``(a11, a21, a22, a31, a32, a33)`` and its inverse
  built like ``SPONGE/MD_core/pbc.hpp:66-101``.

Waters go last, one residue per molecule with masses 16.00/1.008/1.008, so a
solvent module recognises them the way ``solvent_LJ.cpp:193-211`` does.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

CHARGE_SCALE = np.float32(18.2223)
KB = 0.00198716  # kcal/mol/K, SPONGE/common.h CONSTANT_kB
OH_BOND = 0.9572
HOH_ANGLE_DEG = 104.52
Q_O = -0.834
Q_H = 0.417
SIGMA_O = 3.1507
EPS_O = 0.1521
MASS_O = 16.00
MASS_H = 1.008
MASS_SOLUTE = 12.011
# 4-site water (TIP4P, Jorgensen et al. 1983): the negative charge on a
# massless site M on the bisector, 0.15 A from O; LJ on O
OM_DIST_4 = 0.15
Q_H_4 = 0.52
Q_M_4 = -1.04
SIGMA_O_4 = 3.15365
EPS_O_4 = 0.1550


def cell_from_box(a, b, c, alpha=90.0, beta=90.0, gamma=90.0):
    """Lower-triangular cell and inverse, float32, as pbc.hpp:66-101 builds them."""
    f = np.float32
    deg = f(0.0174532925)
    al, be, ga = f(alpha) * deg, f(beta) * deg, f(gamma) * deg
    a, b, c = f(a), f(b), f(c)
    ca, cb, cg = np.cos(al), np.cos(be), np.cos(ga)
    sg = np.sin(ga)
    za = np.sqrt(f(1) - ca * ca - cb * cb - cg * cg + f(2) * ca * cb * cg)
    cell = np.array([a, b * cg, b * sg, c * cb, c / sg * (ca - cb * cg), c / sg * za], dtype=np.float32)
    rcell = np.zeros(6, np.float32)
    rcell[0] = f(1) / cell[0]
    rcell[2] = f(1) / cell[2]
    rcell[5] = f(1) / cell[5]
    rcell[1] = -rcell[0] / np.tan(ga)
    rcell[3] = (ca / np.tan(ga) - cb / sg) / za / a
    rcell[4] = (cb / np.tan(ga) - ca / sg) / za / b
    for k in (1, 3, 4):
        if abs(cell[k]) < 1e-3:
            cell[k] = 0
        if abs(rcell[k]) < 1e-3:
            rcell[k] = 0
    return cell, rcell


def frac_to_cart(s, cell):
    """Row-vector convention r = s * cell (VECTOR * LTMatrix3, vector.hpp:316-321)."""
    a11, a21, a22, a31, a32, a33 = [float(v) for v in cell]
    x = s[:, 0] * a11 + s[:, 1] * a21 + s[:, 2] * a31
    y = s[:, 1] * a22 + s[:, 2] * a32
    z = s[:, 2] * a33
    return np.stack([x, y, z], axis=1)


def get_beta(cutoff, tolerance=1e-5):
    """Ewald screening parameter: erfc(beta*rc)/rc == tol by bisection.

    Restates ``Get_Beta`` (``SPONGE/PM_force/PM_force.cpp:244-272``) in float32.
    """
    f = np.float32
    cutoff = f(cutoff)
    tol = f(tolerance)
    high = f(1.0)
    ihigh = 1
    while True:
        tempf = f(math.erfc(float(high * cutoff))) / cutoff
        if tempf <= tol:
            break
        high = high * f(2)
        ihigh += 1
    ihigh += 50
    low = f(0.0)
    beta = f(0.0)
    for _ in range(1, ihigh):
        beta = (low + high) / f(2)
        tempf = f(math.erfc(float(beta * cutoff))) / cutoff
        if tempf >= tol:
            low = beta
        else:
            high = beta
    return float(beta)


def lj_pair_tables(sigma, eps):
    """Lorentz-Berthelot pair tables in SPONGE's internal triangular form."""
    sigma = np.asarray(sigma, np.float64)
    eps = np.asarray(eps, np.float64)
    t = len(sigma)
    p = t * (t + 1) // 2
    A = np.zeros(p, np.float32)
    B = np.zeros(p, np.float32)
    for a in range(t):
        for b in range(a + 1):
            s = 0.5 * (sigma[a] + sigma[b])
            e = math.sqrt(eps[a] * eps[b])
            idx = a * (a + 1) // 2 + b
            A[idx] = np.float32(4.0 * e * s ** 12) * np.float32(12.0)
            B[idx] = np.float32(4.0 * e * s ** 6) * np.float32(6.0)
    return A, B


def lj_type_index(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    hi = np.maximum(a, b)
    lo = np.minimum(a, b)
    return hi * (hi + 1) // 2 + lo


@dataclass
class System:
    crd: np.ndarray            # (N,3) float32
    charge: np.ndarray         # (N,) float32, scaled
    atom_type: np.ndarray      # (N,) int32
    pair_A: np.ndarray         # (P,) float32 internal
    pair_B: np.ndarray         # (P,) float32 internal
    n_types: int
    excl_start: np.ndarray     # (N,) int32
    excl_numbers: np.ndarray   # (N,) int32
    excl_list: np.ndarray      # (E,) int32
    mass: np.ndarray           # (N,) float32
    res_start: np.ndarray      # (R,) int32
    res_len: np.ndarray        # (R,) int32
    cell: np.ndarray           # (6,) float32
    rcell: np.ndarray          # (6,) float32
    cutoff: float
    skin: float
    beta: float
    vel: np.ndarray = field(default=None)
    n_solute: int = 0
    name: str = ""
    water_points: int = 3      # sites per water residue (3, or 4 with a massless charge site)

    @property
    def n(self):
        return int(self.crd.shape[0])

    @property
    def n_waters(self):
        return (self.n - self.n_solute) // self.water_points

    @property
    def volume(self):
        return float(self.cell[0]) * float(self.cell[2]) * float(self.cell[5])

    @property
    def solvent_atoms(self):
        """Atoms in the trailing run of water residues."""
        return self.water_points * self.n_waters


def _random_rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def _solute_types(rng, n_types=20):
    sig = rng.uniform(2.5, 4.0, n_types)
    eps = np.exp(rng.uniform(math.log(0.02), math.log(0.3), n_types))
    return sig, eps


def water_system(n_waters, box, seed, n_solute=0, cutoff=10.0, skin=2.0,
                 tolerance=1e-5, jitter=0.3, angles=(90.0, 90.0, 90.0),
                 temperature=300.0, n_solute_types=20, name="", solute_types=None, water_points=3):
    """Water (+ optional LJ solute) box on a jittered lattice.

    water_points = 4 makes 4-site waters O, H, H, M (the TIP4P geometry and
    charges, M massless, LJ on O) for the 4-point solvent path.

    Lattice sites fill the box; waters sit on jittered sites with uniformly
    random orientations, solutes (if any) take other sites unjittered, and
    waters crowding a solute are re-jittered until every solute keeps
    0.7*sigma_ij from other solutes and oxygens.
    """
    rng = np.random.default_rng(seed)
    if np.isscalar(box):
        box = (box, box, box)
    cell, rcell = cell_from_box(box[0], box[1], box[2], *angles)
    n_sites_needed = n_waters + n_solute
    m = int(math.ceil(n_sites_needed ** (1.0 / 3.0) - 1e-9))
    while m ** 3 < n_sites_needed:
        m += 1
    sites = rng.choice(m ** 3, size=n_sites_needed, replace=False)
    ijk = np.stack(np.unravel_index(sites, (m, m, m)), axis=1).astype(np.float64)
    frac = (ijk + 0.5) / m
    lattice = frac_to_cart(frac, cell)
    centers = lattice + rng.uniform(-jitter, jitter, size=lattice.shape)
    centers[:n_solute] = lattice[:n_solute]

    sol_sig = sol_eps = None
    if solute_types is not None:
        # a type table shared with other systems (all types present even
        # without solutes, so every such system has the same table)
        sol_sig, sol_eps = solute_types
    elif n_solute:
        sol_sig, sol_eps = _solute_types(rng, n_solute_types)
    if water_points not in (3, 4):
        raise ValueError("water_points must be 3 or 4")
    w4 = water_points == 4
    sigma_all = np.concatenate([[SIGMA_O_4 if w4 else SIGMA_O, 0.0], sol_sig if sol_sig is not None else []])
    eps_all = np.concatenate([[EPS_O_4 if w4 else EPS_O, 0.0], sol_eps if sol_eps is not None else []])
    n_types = len(sigma_all)
    pair_A, pair_B = lj_pair_tables(sigma_all, eps_all)

    sol_center = centers[:n_solute]
    wat_center = centers[n_solute:]
    sol_type = rng.integers(2, n_types, size=n_solute) if n_solute else np.zeros(0, int)
    if n_solute:
        _resolve_solute_overlaps(rng, sol_center, sol_type, wat_center, sigma_all, cell, box, jitter,
                                 sites_wat=lattice[n_solute:])

    # water geometry in its body frame, O at the origin
    half = math.radians(HOH_ANGLE_DEG) / 2
    sites = [[0.0, 0.0, 0.0],
             [OH_BOND * math.sin(half), 0.0, OH_BOND * math.cos(half)],
             [-OH_BOND * math.sin(half), 0.0, OH_BOND * math.cos(half)]]
    if w4:
        sites.append([0.0, 0.0, OM_DIST_4])
    body = np.array(sites)
    R = _random_rotations(rng, n_waters)
    wat = wat_center[:, None, :] + np.einsum("nij,kj->nki", R, body)

    wp = water_points
    n = n_solute + wp * n_waters
    crd = np.empty((n, 3), np.float64)
    crd[:n_solute] = sol_center
    crd[n_solute:] = wat.reshape(-1, 3)
    crd = crd.astype(np.float32)

    charge = np.empty(n, np.float64)
    if n_solute:
        q = rng.normal(0.0, 0.4, n_solute)
        q -= q.mean()
        charge[:n_solute] = q
    charge[n_solute:] = np.tile([0.0, Q_H_4, Q_H_4, Q_M_4] if w4 else [Q_O, Q_H, Q_H], n_waters)
    charge = (charge.astype(np.float32) * CHARGE_SCALE).astype(np.float32)

    atom_type = np.empty(n, np.int32)
    atom_type[:n_solute] = sol_type
    atom_type[n_solute:] = np.tile([0, 1, 1, 1] if w4 else [0, 1, 1], n_waters)

    mass = np.empty(n, np.float32)
    mass[:n_solute] = MASS_SOLUTE
    mass[n_solute:] = np.tile([MASS_O, MASS_H, MASS_H, 0.0] if w4 else [MASS_O, MASS_H, MASS_H], n_waters)

    # exclusions: every intra-water pair (upper triangular)
    excl_numbers = np.zeros(n, np.int32)
    o = n_solute + wp * np.arange(n_waters)
    for k in range(wp - 1):
        excl_numbers[o + k] = wp - 1 - k
    excl_start = np.zeros(n, np.int32)
    excl_start[1:] = np.cumsum(excl_numbers)[:-1]
    excl_list = np.empty(int(excl_numbers.sum()), np.int32)
    for k in range(wp - 1):
        for t, partner in enumerate(range(k + 1, wp)):
            excl_list[excl_start[o + k] + t] = o + partner

    res_len = np.concatenate([np.ones(n_solute, np.int32), np.full(n_waters, wp, np.int32)])
    res_start = np.zeros(len(res_len), np.int32)
    res_start[1:] = np.cumsum(res_len)[:-1]

    vel = (rng.normal(size=(n, 3)) * np.sqrt(KB * temperature / np.maximum(mass, 1e-30))[:, None]).astype(np.float32)
    vel[mass == 0] = 0.0
    return System(crd=crd, charge=charge, atom_type=atom_type, pair_A=pair_A, pair_B=pair_B,
                  n_types=n_types, excl_start=excl_start, excl_numbers=excl_numbers,
                  excl_list=excl_list, mass=mass, res_start=res_start, res_len=res_len,
                  cell=cell, rcell=rcell, cutoff=float(cutoff), skin=float(skin),
                  beta=get_beta(cutoff, tolerance), vel=vel, n_solute=n_solute, name=name,
                  water_points=wp)


def _resolve_solute_overlaps(rng, sol_center, sol_type, wat_center, sigma, cell, box, jitter,
                             sites_sol=None, sites_wat=None, tries=200):
    """Keep every solute at least 0.7*sigma_ij from other solutes and oxygens.

    Solutes sit on their lattice sites without jitter; waters that crowd a
    solute get their jitter redrawn (halved on each retry).  At this site
    density (2.9 A spacing) a 0.7*sigma_ij clearance is the tightest one a
    lattice can always satisfy for sigma up to 4 A.
    """
    from scipy.spatial import cKDTree
    orth = all(abs(float(cell[k])) < 1e-6 for k in (1, 3, 4))
    L = np.array([float(cell[0]), float(cell[2]), float(cell[5])])
    ns = len(sol_center)
    amp = np.full(len(wat_center), jitter)
    for _ in range(tries):
        pts = np.concatenate([sol_center, wat_center])
        typ = np.concatenate([sol_type, np.zeros(len(wat_center), int)])
        if orth:
            tree = cKDTree(np.mod(pts, L), boxsize=L)
        else:
            tree = cKDTree(pts)
        pairs = tree.query_pairs(0.7 * 4.0, output_type="ndarray")
        if len(pairs) == 0:
            return
        pairs = pairs[(pairs[:, 0] < ns) | (pairs[:, 1] < ns)]
        d = pts[pairs[:, 0]] - pts[pairs[:, 1]]
        if orth:
            d -= np.round(d / L) * L
        r = np.linalg.norm(d, axis=1)
        sij = 0.5 * (sigma[typ[pairs[:, 0]]] + sigma[typ[pairs[:, 1]]])
        bad = pairs[r < 0.7 * sij]
        if len(bad) == 0:
            return
        w = np.unique(bad.ravel())
        w = w[w >= ns] - ns
        if len(w) == 0:
            raise RuntimeError("solute-solute clearance impossible at this density")
        amp[w] *= 0.5
        wat_center[w] = sites_wat[w] + rng.uniform(-1, 1, size=(len(w), 3)) * amp[w, None]
    raise RuntimeError("could not place solutes without overlaps")


# ---------------------------------------------------------------------------
# Named workloads.  Sizes follow the workload descriptions: a 40 A box of
# 2,160 waters; a 96,000-atom mixed box; a ~1.0M-atom water box; 256 uneven
# systems; a Poisson stream of MD segments.
# ---------------------------------------------------------------------------

def water_box_6480(seed=1):
    return water_system(2160, 40.0, seed, cutoff=10.0, skin=2.0, name="water-6480")


def mixed_box_96k(seed=2):
    # 30,000 waters + 6,000 solute atoms in a 99 A cubic box (0.0989 atoms/A^3)
    return water_system(30000, 99.0, seed, n_solute=6000, cutoff=10.0, skin=2.0, name="mixed-96k")


def water_box_1m(seed=3):
    n_w = 333333
    L = (n_w / 0.0334) ** (1.0 / 3.0)
    return water_system(n_w, L, seed, cutoff=12.0, skin=2.0, name="water-1m")


def batch_systems(n_systems=256, seed=4, n_min=1500, n_max=24000, skin=2.0):
    """Independent systems with log-uniform atom counts and uneven cutoffs.

    The cutoff is drawn uniformly from {8, 10, 12} among the values that keep
    rc + skin <= L/2, so each pair has a single minimum image.
    """
    rng = np.random.default_rng(seed)
    # one solute type table for the whole batch
    types = shared_solute_types(seed)
    out = []
    for k in range(n_systems):
        n_atoms = int(math.exp(rng.uniform(math.log(n_min), math.log(n_max))))
        frac_sol = rng.uniform(0.0, 0.15)
        n_sol = int(round(frac_sol * n_atoms))
        n_w = max(1, (n_atoms - n_sol) // 3)
        L = ((n_w + n_sol) / 0.0334) ** (1.0 / 3.0)
        allowed = [rc for rc in (8.0, 10.0, 12.0) if rc + skin <= L / 2]
        if not allowed:
            allowed = [max(4.0, L / 2 - skin)]
        rc = float(rng.choice(allowed))
        out.append(water_system(n_w, L, int(rng.integers(1 << 31)), n_solute=n_sol, cutoff=rc,
                                skin=skin, name=f"batch-{k}", solute_types=types))
    return out


@dataclass
class Request:
    rid: int
    arrival_s: float
    n_atoms: int
    steps: int
    seed: int


def request_stream(duration_s=600.0, rate_per_s=40.0, seed=5, n_min=1000, n_max=50000,
                   steps_min=500, steps_max=5000):
    """Poisson arrivals of MD segments with log-uniform sizes."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    rid = 0
    while True:
        t += rng.exponential(1.0 / rate_per_s)
        if t > duration_s:
            break
        n_atoms = int(math.exp(rng.uniform(math.log(n_min), math.log(n_max))))
        steps = int(rng.integers(steps_min, steps_max + 1))
        out.append(Request(rid, t, n_atoms, steps, int(rng.integers(1 << 31))))
        rid += 1
    return out


def shared_solute_types(seed=4):
    """The one solute type table of the batched and served workloads."""
    return _solute_types(np.random.default_rng(seed + 1000), 20)


def request_system(req: Request, skin=2.0):
    rng = np.random.default_rng(req.seed)
    frac_sol = rng.uniform(0.0, 0.15)
    n_sol = int(round(frac_sol * req.n_atoms))
    n_w = max(1, (req.n_atoms - n_sol) // 3)
    L = ((n_w + n_sol) / 0.0334) ** (1.0 / 3.0)
    allowed = [rc for rc in (8.0, 10.0, 12.0) if rc + skin <= L / 2]
    if not allowed:
        allowed = [max(4.0, L / 2 - skin)]
    rc = float(rng.choice(allowed))
    # a small box can draw a solute arrangement the lattice cannot clear:
    # draw the placement again (deterministically) until one fits
    for attempt in range(50):
        try:
            return water_system(n_w, L, int(rng.integers(1 << 31)), n_solute=n_sol, cutoff=rc, skin=skin,
                                name=f"req-{req.rid}", solute_types=shared_solute_types())
        except RuntimeError:
            if attempt == 49:
                raise


# ---------------------------------------------------------------------------
# Two-state (alchemical) variants for LJ_SOFT_CORE
# ---------------------------------------------------------------------------

@dataclass
class FepSystem:
    """A two-state copy of a System: per-atom state-A / state-B LJ types, the
    four triangular tables (AA, AB of state A; BA, BB of state B, internal
    convention), state charges, and the soft-core parameters
    (lambda_lj, soft_core_alpha, soft_core_powfer, soft_core_sigma,
    soft_core_sigma_min)."""
    base: System
    type_a: np.ndarray
    type_b: np.ndarray
    n_types_a: int
    n_types_b: int
    AA: np.ndarray
    AB: np.ndarray
    BA: np.ndarray
    BB: np.ndarray
    charge_a: np.ndarray
    charge_b: np.ndarray
    lam: float
    alpha: float = 0.5
    p: float = 1.0
    sigma: float = 3.0
    sigma_min: float = 0.0
    changed: np.ndarray = field(default=None)   # the atoms the generator perturbed

    def charge(self, lam=None):
        """Charges at lambda, q = (1 - lambda) q_A + lambda q_B (float32)."""
        lam = self.lam if lam is None else lam
        return ((1.0 - lam) * self.charge_a.astype(np.float64) +
                lam * self.charge_b.astype(np.float64)).astype(np.float32)

    def charge_ba(self):
        return (self.charge_b.astype(np.float64) - self.charge_a.astype(np.float64)).astype(np.float32)

    def params(self, lam=None):
        return np.array([self.lam if lam is None else lam, self.alpha, self.p, self.sigma, self.sigma_min],
                        np.float32)

    def system(self, lam=None):
        """The base System with the charges at lambda."""
        from dataclasses import replace
        return replace(self.base, charge=self.charge(lam))

    def controller(self, lam=None):
        return {"lambda_lj": float(self.lam if lam is None else lam), "soft_core_alpha": self.alpha,
                "soft_core_powfer": self.p, "soft_core_sigma": self.sigma, "soft_core_sigma_min": self.sigma_min}


def _with_dummy_type(A, B, n_types):
    """Tables of n_types + 1 types, the last one interacting with nothing."""
    m = n_types + 1
    A2 = np.zeros(m * (m + 1) // 2, np.float32)
    B2 = np.zeros_like(A2)
    A2[:len(A)] = A
    B2[:len(B)] = B
    return A2, B2


def _permute_table(T, perm):
    """Table re-indexed so that new type perm[t] is old type t."""
    m = len(perm)
    out = np.zeros_like(T)
    for a in range(m):
        for b in range(a + 1):
            out[lj_type_index(perm[a], perm[b])] = T[lj_type_index(a, b)]
    return out


def fep_system(base: System, n_perturbed=24, seed=7, lam=0.5, alpha=0.5, p=1.0, sigma=3.0, sigma_min=0.0,
               kinds=("vanish", "appear", "mutate"), permute_b=True, bond_perturbed=True):
    """Perturbs the n_perturbed solutes nearest a random solute (a ligand):
    "vanish" atoms lose their LJ type (a dummy type that interacts with
    nothing) and charge in state B, "appear" atoms have them only in state
    B, "mutate" atoms take another solute type and the opposite half charge.
    permute_b renumbers state B's types (its own index space, as the
    reference allows); bond_perturbed adds exclusions between consecutive
    perturbed atoms closer than 5 A, so excluded pairs run through the
    perturbed set too."""
    if base.n_solute < n_perturbed:
        raise ValueError("not enough solute atoms to perturb")
    rng = np.random.default_rng(seed)
    T = base.n_types
    dummy = T
    AA, AB = _with_dummy_type(base.pair_A, base.pair_B, T)
    BA, BB = AA.copy(), AB.copy()
    # the ligand: solutes nearest a random one (minimum image in fractional space)
    c0 = int(rng.integers(base.n_solute))
    sol = base.crd[:base.n_solute].astype(np.float64)
    r = np.asarray(base.rcell, np.float64)
    c = np.asarray(base.cell, np.float64)
    d = sol - sol[c0]
    fx = d[:, 0] * r[0] + d[:, 1] * r[1] + d[:, 2] * r[3]
    fy = d[:, 1] * r[2] + d[:, 2] * r[4]
    fz = d[:, 2] * r[5]
    fx -= np.round(fx)
    fy -= np.round(fy)
    fz -= np.round(fz)
    dist = np.sqrt((fx * c[0] + fy * c[1] + fz * c[3]) ** 2 + (fy * c[2] + fz * c[4]) ** 2 + (fz * c[5]) ** 2)
    chosen = np.sort(np.argsort(dist, kind="stable")[:n_perturbed])
    ta = base.atom_type.astype(np.int32).copy()
    tb = ta.copy()
    qa = base.charge.astype(np.float32).copy()
    qb = qa.copy()
    n_solute_types = T - 2
    for k, a in enumerate(chosen):
        kind = kinds[k % len(kinds)]
        if kind == "vanish":
            tb[a] = dummy
            qb[a] = 0.0
        elif kind == "appear":
            ta[a] = dummy
            qa[a] = 0.0
        elif kind == "mutate":
            old = int(ta[a]) - 2
            tb[a] = 2 + (old + 1 + int(rng.integers(n_solute_types - 1))) % n_solute_types
            qb[a] = np.float32(-0.5) * qa[a]
        else:
            raise ValueError(kind)
    n_b = T + 1
    if permute_b:
        perm = rng.permutation(n_b)
        BA, BB = _permute_table(BA, perm), _permute_table(BB, perm)
        tb = perm[tb].astype(np.int32)
    s = base
    if bond_perturbed and len(chosen) > 1:
        # each perturbed atom bonded to its nearest perturbed neighbour within 5 A
        g = base.crd[chosen].astype(np.float64)
        dd = g[:, None, :] - g[None, :, :]
        f0 = dd[..., 0] * r[0] + dd[..., 1] * r[1] + dd[..., 2] * r[3]
        f1 = dd[..., 1] * r[2] + dd[..., 2] * r[4]
        f2 = dd[..., 2] * r[5]
        f0 -= np.round(f0)
        f1 -= np.round(f1)
        f2 -= np.round(f2)
        dm = np.sqrt((f0 * c[0] + f1 * c[1] + f2 * c[3]) ** 2 + (f1 * c[2] + f2 * c[4]) ** 2 + (f2 * c[5]) ** 2)
        np.fill_diagonal(dm, np.inf)
        pairs = set()
        for k in range(len(chosen)):
            m = int(np.argmin(dm[k]))
            if dm[k, m] < 5.0:
                u, v = int(chosen[k]), int(chosen[m])
                pairs.add((min(u, v), max(u, v)))
        if pairs:
            lists = [list(base.excl_list[base.excl_start[i]:base.excl_start[i] + base.excl_numbers[i]])
                     for i in range(base.n)]
            for lo, hi in pairs:
                lists[lo].append(hi)
            num = np.array([len(x) for x in lists], np.int32)
            start = np.zeros(base.n, np.int32)
            start[1:] = np.cumsum(num)[:-1]
            flat = np.array([j for x in lists for j in sorted(x)], np.int32)
            from dataclasses import replace
            s = replace(base, excl_start=start, excl_numbers=num, excl_list=flat)
    return FepSystem(base=s, type_a=ta, type_b=tb, n_types_a=T + 1, n_types_b=n_b, AA=AA, AB=AB, BA=BA, BB=BB,
                     charge_a=qa, charge_b=qb, lam=_f32(lam), alpha=_f32(alpha), p=_f32(p), sigma=_f32(sigma),
                     sigma_min=_f32(sigma_min), changed=chosen)


def _f32(v):
    """A parameter as the float32 value the modules receive."""
    return float(np.float32(v))
