"""System specifications and the synthetic workloads.

`SystemSpec` is plain host data with the fields of the C `scmf_spec`: box,
grid, interaction matrix xn[t + n*s] (diagonal kappaN, off-diagonal chiN, as
Phase_info_gpu::xn, init_config.cu:670-672), reference chain length N_ref,
harmonic bond constant k, smart-MC step A, the Philox seed, the Hamiltonian,
the field rule and the count width, plus one `Arch` per polymer
architecture (chain length, chain count, monomer type per bead, bonds,
initial bond sigma).

The workload generators build the synthetic systems the benchmark and tests
run: a plain AB diblock melt, a large diblock melt, a homopolymer blend with a
diblock compatibiliser, a mix of uneven diblock systems for batching, and
random requests for serving.  Unit choice for the synthetic systems (cell
units, cell edge 1): k = 3 / (2 b^2) with b = 0.7, initial per-component bond
sigma b / sqrt(3) (so k = 1 / (2 sigma^2) as in init_config.cu:480-484),
A = 0.5, R = sqrt(2A), omega carrying the 1/N_ref factor of the reference's
SCMF0 field.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

from . import _lib
from ._lib import FIELD_EVERY, FIELD_REFERENCE, HAM_SCMF0, check, lib


@dataclass
class Arch:
    length: int
    n_chains: int
    mono_type: Sequence[int]
    bonds: Sequence[Sequence[int]]
    init_sigma: float = 0.0


@dataclass
class SystemSpec:
    n_types: int
    nx: int
    ny: int
    nz: int
    lx: float
    ly: float
    lz: float
    xn: Sequence[float]                # flat [t + n*s]
    nref: int
    harmonic_normb: float
    smc_a: float
    seed: int = 0
    hamiltonian: int = HAM_SCMF0
    field_rule: int = FIELD_EVERY
    count_bits: int = 32
    archs: List[Arch] = field(default_factory=list)

    @property
    def n_beads(self) -> int:
        return sum(a.length * a.n_chains for a in self.archs)

    @property
    def n_chains(self) -> int:
        return sum(a.n_chains for a in self.archs)

    @property
    def n_cells(self) -> int:
        return self.nx * self.ny * self.nz

    def to_c(self) -> C.c_void_p:
        """A new C scmf_spec handle (caller destroys with scmf_spec_destroy)."""
        L = lib()
        h = C.c_void_p()
        check(L.scmf_spec_create(self.n_types, self.nx, self.ny, self.nz, self.lx, self.ly, self.lz, C.byref(h)))
        try:
            xn = np.ascontiguousarray(self.xn, dtype=np.float64)
            check(L.scmf_spec_set_xn(h, xn.ctypes.data_as(C.POINTER(C.c_double)), self.n_types))
            p = _lib.Params(self.nref, self.harmonic_normb, self.smc_a, self.seed & (2**64 - 1), self.hamiltonian,
                            self.field_rule, self.count_bits, 0)
            check(L.scmf_spec_set_params(h, C.byref(p)))
            for a in self.archs:
                mt = np.ascontiguousarray(a.mono_type, dtype=np.int32)
                bd = np.ascontiguousarray(np.asarray(a.bonds, dtype=np.int32).reshape(-1))
                check(L.scmf_spec_add_arch(h, a.length, a.n_chains, mt.ctypes.data_as(C.POINTER(C.c_int32)),
                                           len(bd) // 2, bd.ctypes.data_as(C.POINTER(C.c_int32)), a.init_sigma))
        except Exception:
            L.scmf_spec_destroy(h)
            raise
        return h

    @staticmethod
    def from_c(h) -> "SystemSpec":
        L = lib()
        info = _lib.SpecInfo()
        check(L.scmf_spec_get_info(h, C.byref(info)))
        p = _lib.Params()
        check(L.scmf_spec_get_params(h, C.byref(p)))
        n = info.n_types
        xn = np.zeros(n * n, dtype=np.float64)
        check(L.scmf_spec_get_xn(h, xn.ctypes.data_as(C.POINTER(C.c_double)), n))
        archs = []
        for i in range(info.n_arch):
            length, nch, nb = C.c_int32(), C.c_int32(), C.c_int32()
            sig = C.c_double()
            check(L.scmf_spec_get_arch(h, i, C.byref(length), C.byref(nch), None, 0, None, 0, C.byref(nb), C.byref(sig)))
            mt = np.zeros(length.value, dtype=np.int32)
            bd = np.zeros(max(1, 2 * nb.value), dtype=np.int32)
            check(L.scmf_spec_get_arch(h, i, None, None, mt.ctypes.data_as(C.POINTER(C.c_int32)), length.value,
                                       bd.ctypes.data_as(C.POINTER(C.c_int32)), 2 * nb.value, None, None))
            archs.append(Arch(length.value, nch.value, mt.tolist(), bd[:2 * nb.value].reshape(-1, 2).tolist(), sig.value))
        return SystemSpec(n, info.nx, info.ny, info.nz, info.lx, info.ly, info.lz, xn.tolist(), p.reference_nbeads,
                          p.harmonic_normb, p.smc_a, p.seed, p.hamiltonian, p.field_rule, p.count_bits, archs)

    @staticmethod
    def from_files(configuration_dat: str, polymer_dat: str, seed: int) -> "SystemSpec":
        """Parse the reference's input files through the library's parsers."""
        L = lib()
        h = C.c_void_p()
        check(L.scmf_spec_load_files(configuration_dat.encode(), polymer_dat.encode(), seed, C.byref(h)))
        try:
            return SystemSpec.from_c(h)
        finally:
            L.scmf_spec_destroy(h)

    def device_bytes(self) -> int:
        """Device memory a system of this spec holds (approximate, upper bound)."""
        beads, cells = self.n_beads, self.n_cells * self.n_types
        cb = (cells + 1) // 2 * 4 if self.count_bits == 16 else cells * 4
        return 3 * (beads + 4) * 4 + self.n_chains * 4 + 2 * cb + cells * 4 + 256 * 1024


# ------------------------------------------------------------- workloads

def interaction_matrix(n_types: int, chi_n: float, kappa_n: float) -> List[float]:
    xn = np.full((n_types, n_types), chi_n, dtype=np.float64)
    np.fill_diagonal(xn, kappa_n)
    return xn.reshape(-1).tolist()


def linear_bonds(n: int) -> List[List[int]]:
    return [[i, i + 1] for i in range(n - 1)]


def diblock_arch(n: int, f_a: float, n_chains: int, sigma: float) -> Arch:
    na = int(round(f_a * n))
    return Arch(n, n_chains, [0] * na + [1] * (n - na), linear_bonds(n), sigma)


def homopolymer_arch(n: int, t: int, n_chains: int, sigma: float) -> Arch:
    return Arch(n, n_chains, [t] * n, linear_bonds(n), sigma)


def cell_units(b: float = 0.7):
    """k = 3/(2 b^2) and the per-component initial bond sigma b/sqrt(3)."""
    return 3.0 / (2.0 * b * b), b / math.sqrt(3.0)


def diblock_melt(n_chains: int, n: int, f_a: float, grid, chi_n: float, kappa_n: float = 50.0, seed: int = 42,
                 b: float = 0.7, smc_a: float = 0.5, field_rule: int = FIELD_EVERY, count_bits: int = 32,
                 nref: int | None = None) -> SystemSpec:
    nx, ny, nz = grid
    k, sig = cell_units(b)
    return SystemSpec(2, nx, ny, nz, float(nx), float(ny), float(nz), interaction_matrix(2, chi_n, kappa_n),
                      nref or n, k, smc_a, seed, HAM_SCMF0, field_rule, count_bits,
                      [diblock_arch(n, f_a, n_chains, sig)])


def plain_system(seed: int = 42) -> SystemSpec:
    """1,000 AB diblocks, N=32, f_A=0.5, 16^3 cells, chiN=20, kappaN=50, 16-bit counts."""
    return diblock_melt(1000, 32, 0.5, (16, 16, 16), 20.0, 50.0, seed, count_bits=16)


def large_system(seed: int = 7, scale: float = 1.0) -> SystemSpec:
    """1.6M AB diblocks, N=32 (51.2M beads), f_A=0.3, 128^3 cells, chiN=25, kappaN=50.
    `scale` < 1 shrinks chains and grid together (same density) for tests."""
    if scale == 1.0:
        return diblock_melt(1_600_000, 32, 0.3, (128, 128, 128), 25.0, 50.0, seed)
    edge = max(8, int(round(128 * scale ** (1 / 3))))
    chains = int(round(1_600_000 * edge ** 3 / 128 ** 3))
    return diblock_melt(chains, 32, 0.3, (edge, edge, edge), 25.0, 50.0, seed)


def blend_system(seed: int = 11, n_chains: int = 2_000_000, grid=(256, 256, 64)) -> SystemSpec:
    """50% A-homopolymer N=64, 40% B-homopolymer N=64, 10% AB diblock N=32 in one
    system; chiN=15 referenced to N=64, kappaN=40."""
    k, sig = cell_units()
    na, nb = n_chains // 2, (n_chains * 2) // 5
    nd = n_chains - na - nb
    nx, ny, nz = grid
    return SystemSpec(2, nx, ny, nz, float(nx), float(ny), float(nz), interaction_matrix(2, 15.0, 40.0), 64, k, 0.5,
                      seed, HAM_SCMF0, FIELD_EVERY, 32,
                      [homopolymer_arch(64, 0, na, sig), homopolymer_arch(64, 1, nb, sig), diblock_arch(32, 0.5, nd, sig)])


BATCH_EDGES = (16, 24, 32, 48, 64)
BATCH_LENGTHS = (16, 32, 48, 64)


def batched_mix(n_systems: int = 256, mix_seed: int = 2024, edge_scale: float = 1.0) -> List[SystemSpec]:
    """Uneven diblock systems: per-axis edge from {16,24,32,48,64}, N from
    {16,32,48,64}, f_A ~ U[0.2,0.8], chiN ~ U[10,30], kappaN = 50, chains =
    round(7.8 cells / N), Philox seed 1000+i, field update every sweep."""
    rng = np.random.default_rng(mix_seed)
    out = []
    for i in range(n_systems):
        edges = [max(4, int(round(e * edge_scale))) for e in rng.choice(BATCH_EDGES, 3)]
        n = int(rng.choice(BATCH_LENGTHS))
        f_a = float(rng.uniform(0.2, 0.8))
        chi = float(rng.uniform(10.0, 30.0))
        cells = edges[0] * edges[1] * edges[2]
        chains = max(1, int(round(7.8 * cells / n)))
        out.append(diblock_melt(chains, n, f_a, edges, chi, 50.0, 1000 + i))
    return out


def served_request(rng: np.random.Generator, seed: int, edge_lo: int = 16, edge_hi: int = 128):
    """One request: a diblock chiN-sweep system as in the batched mix but with
    per-axis edge log-uniform in [16, 128], and K sweeps from {50, 100, 500}."""
    edges = [int(round(math.exp(rng.uniform(math.log(edge_lo), math.log(edge_hi))))) for _ in range(3)]
    n = int(rng.choice(BATCH_LENGTHS))
    f_a = float(rng.uniform(0.2, 0.8))
    chi = float(rng.uniform(10.0, 30.0))
    cells = edges[0] * edges[1] * edges[2]
    chains = max(1, int(round(7.8 * cells / n)))
    k_sweeps = int(rng.choice((50, 100, 500)))
    return diblock_melt(chains, n, f_a, edges, chi, 50.0, seed), k_sweeps
