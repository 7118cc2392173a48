"""Seeded synthetic (T) inputs in the reference's memory layouts.

The reference reads its inputs from a ``triples.restart`` file written by GAMESS
after CCSD (``src/triples-ijk/program.F90:195-223``).  The real integrals of the
published water / Ar6 runs are not available, so these generators stand in for
them, with the shapes, symmetries and value distributions of the five workloads:

* ``water-avdz``  no=4,  nu=36,  seed 0   (water aug-cc-pVDZ shape)
* ``no16-nu200``  no=16, nu=200, seed 1
* ``no24-nu320``  no=24, nu=320, seed 2, log-uniform magnitudes in [1e-6, 1]
* ``batch96``     96 systems, seeds 100+s, no~U{3..12}, nu~U{24..140}
* ``no12-nu120``  no=12, nu=120, seed 3   (gradient workload)

Every array is returned as a flat float64 vector in the Fortran column-major
order the reference uses (first index fastest):

========  ==================  =========================================
name      Fortran shape       meaning
========  ==================  =========================================
eh        (no)                occupied orbital energies
ep        (nu)                virtual orbital energies
t1        (no, nu)            T1 amplitudes, file layout
t2        (nu, nu, no, no)    T2(a,b,i,j), T2(a,b,i,j) = T2(b,a,j,i)
vm        (no, nu, no, no)    VM(l,c,x,y) = (c x | l y)        [VOOO]
voe       (nu, nu, no, no)    VOE(a,b,i,j) = (a i | b j)       [VVOO]
vvvo      (nutr, nu*no)       packed (a b | c x): column x*nu+c holds the
                              a>=b triangle, row-packed as in CPYTSQ
========  ==================  =========================================

(``common_cc.f90:4-16`` for the dimensions, ``common_functions.f:43-60`` for the
triangle packing, ``triples_cpu.F90:633-636`` for the VM l<->y symmetry.)
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class TriplesInputs:
    no: int
    nu: int
    eh: np.ndarray
    ep: np.ndarray
    t1: np.ndarray
    t2: np.ndarray
    vm: np.ndarray
    voe: np.ndarray
    vvvo: np.ndarray
    name: str = ""
    seed: int = 0

    @property
    def nutr(self) -> int:
        return self.nu * (self.nu + 1) // 2

    def arrays(self):
        return (self.eh, self.ep, self.t1, self.t2, self.vm, self.voe, self.vvvo)

    def nbytes(self) -> int:
        return sum(a.nbytes for a in self.arrays())


WORKLOADS = {
    "water-avdz": dict(no=4, nu=36, seed=0, dist="normal"),
    "no16-nu200": dict(no=16, nu=200, seed=1, dist="normal"),
    "no24-nu320": dict(no=24, nu=320, seed=2, dist="log"),
    "no12-nu120": dict(no=12, nu=120, seed=3, dist="normal"),
}


def _draw(rng: np.random.Generator, shape, dist: str, sigma: float) -> np.ndarray:
    if dist == "normal":
        return rng.normal(0.0, sigma, size=shape)
    if dist == "log":
        mag = 10.0 ** rng.uniform(-6.0, 0.0, size=shape)
        sign = np.where(rng.random(size=shape) < 0.5, -1.0, 1.0)
        return mag * sign
    raise ValueError(f"unknown distribution {dist!r}")


def _pair_mirror(x: np.ndarray, no: int) -> np.ndarray:
    """Make X[a,b,i,j] = X[b,a,j,i] by copying the (a,i) <= (b,j) half."""
    nu = x.shape[0]
    key = np.arange(nu)[:, None] * no + np.arange(no)[None, :]  # key[a,i]
    k1 = key[:, None, :, None]  # (a,i) -> broadcast over [a,b,i,j]
    k2 = key[None, :, None, :]  # (b,j)
    swapped = x.transpose(1, 0, 3, 2)
    return np.where(k1 <= k2, x, swapped)


def generate(no: int, nu: int, seed: int, dist: str = "normal", name: str = "") -> TriplesInputs:
    """Draw one system.  Draw order is fixed so a seed always gives the same bytes."""
    if no < 1 or nu < 1:
        raise ValueError("no and nu must be positive")
    rng = np.random.default_rng(seed)
    eh = np.sort(rng.uniform(-1.4, -0.4, size=no))
    ep = np.sort(rng.uniform(0.1, 4.0, size=nu))
    t1m = rng.normal(0.0, 0.005, size=(no, nu))                       # T1[i,a]
    # T2[a,b,i,j] = X / (e_a + e_b - e_i - e_j), X symmetric under (a,i)<->(b,j)
    x = _pair_mirror(_draw(rng, (nu, nu, no, no), dist, 0.05), no)
    den = ep[:, None, None, None] + ep[None, :, None, None] - eh[None, None, :, None] - eh[None, None, None, :]
    t2m = x / den
    del x, den
    # VVVO[a,b,c,x] = (ab|cx), symmetric a<->b: draw the packed a>=b triangle directly
    nutr = nu * (nu + 1) // 2
    vvvo = _draw(rng, (nu * no, nutr), dist, 0.05)                    # [column][packed row]
    # VOOO[a,i,j,k] = (ai|jk), symmetric j<->k
    vooo = _draw(rng, (nu, no, no, no), dist, 0.05)
    jj = np.arange(no)
    upper = (jj[:, None] <= jj[None, :])[None, None, :, :]
    vooo = np.where(upper, vooo, vooo.transpose(0, 1, 3, 2))
    # VVOO[a,b,i,j] = (ai|bj), symmetric (a,i)<->(b,j)
    vvoo = _pair_mirror(_draw(rng, (nu, nu, no, no), dist, 0.05), no)
    # reference layouts (Fortran order == C order of the reversed index tuple)
    t1 = np.ascontiguousarray(t1m.T).ravel()                           # t1(no,nu): [a][i]
    t2 = np.ascontiguousarray(t2m.transpose(3, 2, 1, 0)).ravel()       # T2(a,b,i,j)
    del t2m
    vmm = vooo.transpose(2, 0, 1, 3)                                   # VM[l,c,x,y] = VOOO[c,x,l,y]
    vm = np.ascontiguousarray(vmm.transpose(3, 2, 1, 0)).ravel()
    voe = np.ascontiguousarray(vvoo.transpose(3, 2, 1, 0)).ravel()
    return TriplesInputs(no=no, nu=nu, eh=eh, ep=ep, t1=t1, t2=t2, vm=vm, voe=voe,
                         vvvo=vvvo.ravel(), name=name or f"no{no}-nu{nu}-s{seed}", seed=seed)


def with_decay(inp: TriplesInputs, bits_per_index: float) -> TriplesInputs:
    """A copy of ``inp`` whose magnitudes fall by 2^-bits_per_index per virtual
    index, like integrals over localised orbitals ordered by distance: every
    entry is scaled by g(a) = 2^(-bits_per_index * a) for each virtual index a
    it carries (T1, T2, VM, VOE, VVVO).  Energies stay finite; W tiles then
    span many binary orders of magnitude, which the per-tile digit count of the
    emulated form exploits."""
    no, nu = inp.no, inp.nu
    g = 2.0 ** (-bits_per_index * np.arange(nu))
    t1 = (inp.t1.reshape(nu, no) * g[:, None]).ravel()
    t2 = (inp.t2.reshape(no, no, nu, nu) * g[None, None, :, None] * g[None, None, None, :]).ravel()
    vm = (inp.vm.reshape(no, no, nu, no) * g[None, None, :, None]).ravel()
    voe = (inp.voe.reshape(no, no, nu, nu) * g[None, None, :, None] * g[None, None, None, :]).ravel()
    ii = np.arange(nu)
    I, J = np.meshgrid(ii, ii, indexing="ij")
    low = I >= J
    gp = np.zeros(nu * (nu + 1) // 2)
    gp[(I * (I + 1) // 2 + J)[low]] = (g[:, None] * g[None, :])[low]      # packed (I >= J)
    col = np.tile(g, no)                                                  # column x*nu + r1 -> g(r1)
    vvvo = (inp.vvvo.reshape(nu * no, -1) * col[:, None] * gp[None, :]).ravel()
    return TriplesInputs(no=no, nu=nu, eh=inp.eh.copy(), ep=inp.ep.copy(), t1=t1, t2=t2, vm=vm, voe=voe,
                         vvvo=vvvo, name=f"{inp.name}-decay{bits_per_index:g}", seed=inp.seed)


def workload(name: str) -> TriplesInputs:
    """One of the named single-system workloads."""
    cfg = WORKLOADS[name]
    return generate(cfg["no"], cfg["nu"], cfg["seed"], cfg["dist"], name=name)


def batch96_shapes(count: int = 96):
    """(no, nu, seed) of the batched workload: system s uses seed 100+s."""
    out = []
    for s in range(count):
        rng = np.random.default_rng(100 + s)
        no = int(rng.integers(3, 13))
        nu = int(rng.integers(24, 141))
        out.append((no, nu, 100 + s))
    return out


def batch96(count: int = 96):
    """The 96 uneven systems of the batched workload (normal distributions).
    A fresh generator on seed 100+s first draws (no, nu), then the system's
    arrays are drawn from another fresh generator on the same seed."""
    return [generate(no, nu, seed, "normal", name=f"batch-s{seed - 100}")
            for (no, nu, seed) in batch96_shapes(count)]


def flops(no: int, nu: int) -> float:
    """Algorithmic flops of one (T) evaluation: 12 nu^3 (no+nu) per i>j>k tuple and
    half that per degenerate tuple (``ijk_tuple.f90:19-28``), i.e.
    2 nu^3 (no+nu) (no^3 - no)."""
    return 2.0 * nu ** 3 * (no + nu) * (no ** 3 - no)


def tuple_counts(no: int):
    """(ijk, iij, ijj) tuple counts (``triples.F90:51-53``)."""
    return no * (no - 1) * (no - 2) // 6, no * (no - 1) // 2, no * (no - 1) // 2
