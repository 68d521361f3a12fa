"""Host mirror of jaxqft.fermions.wilson.WilsonDiracOperator's bookkeeping.

The operator itself (D, D^dag, D^dag D) runs in libwilson_sm100 and is reached
through SU3WilsonNf2.apply_* or WilsonContext.apply; what callers also read
from the reference's operator object is its floating-point operation count,
used to report GFLOP/s (jaxqft/fermions/wilson.py:349-437, consumed by
models/su3_wilson_nf2.py:1780-1795 and scripts/wilson/bench_wilson_matrix.py).
The count is a convention, not a measurement, so the formula is the
reference's, term for term: per direction two projected hops (colour multiply
of all Ns spin rows + spin projection) and the output accumulation; the
sparse-gamma form counts one complex phase multiply per spin-colour entry.
For Nc = 3 it gives 3552 flops per site for the hopping term and 3600 with the
diagonal (mass) term.
"""

from __future__ import annotations


class WilsonDiracOperator:
    """The reference operator's parameters (wilson.py:18-48: ndim, mass,
    wilson_r, gamma) and its flop counter.  Ns is the gamma matrices' size,
    2^(ndim // 2) for the Euclidean basis of fermions/gamma.py."""

    def __init__(self, ndim: int = 4, mass: float = 0.0, wilson_r: float = 1.0, dtype=None, gamma=None,
                 use_half_spinor: bool = False):
        self.ndim = int(ndim)
        self.Nd = self.ndim
        if self.Nd < 1:
            raise ValueError("ndim must be >= 1")
        self.mass = float(mass)
        self.wilson_r = float(wilson_r)
        self.dtype = dtype
        self.gamma = gamma
        self.use_half_spinor = bool(use_half_spinor)
        self.Ns = int(gamma.shape[-1]) if gamma is not None else 2 ** (self.Nd // 2)

    def flops_per_site_dslash(self, nc: int, use_sparse_gamma: bool = True, complex_mul_flops: int = 6,
                              complex_add_flops: int = 2, real_complex_mul_flops: int = 2) -> int:
        """Flops per site of the hopping term (wilson.py:349-389)."""
        nc = int(nc)
        if nc < 1:
            raise ValueError("nc must be >= 1")
        ns, nd = self.Ns, self.Nd
        cm, ca, rm = int(complex_mul_flops), int(complex_add_flops), int(real_complex_mul_flops)
        color = ns * nc * (cm * nc + ca * (nc - 1))      # Nc x Nc times Nc, every spin row
        if use_sparse_gamma:
            gamma = ns * nc * cm                          # one phase multiply per entry
        else:
            gamma = nc * ns * (cm * ns + ca * (ns - 1))   # dense Ns x Ns per colour
        project = gamma + ns * nc * (2 * rm + ca)         # r psi + coeff gamma psi
        accum = ns * nc * (2 * ca + rm)                   # out += -1/2 (fwd + bwd)
        return int(nd * (2 * (color + project) + accum))

    def flops_per_site_matvec(self, nc: int, use_sparse_gamma: bool = True, include_diagonal: bool = True,
                              complex_mul_flops: int = 6, complex_add_flops: int = 2,
                              real_complex_mul_flops: int = 2) -> int:
        """Flops per site of D = diagonal + hopping term (wilson.py:391-415)."""
        d = self.flops_per_site_dslash(nc, use_sparse_gamma, complex_mul_flops, complex_add_flops,
                                       real_complex_mul_flops)
        if not include_diagonal:
            return int(d)
        return int(d + self.Ns * int(nc) * (int(real_complex_mul_flops) + int(complex_add_flops)))

    def flops_per_matvec_call(self, nc: int, volume: int, batch: int = 1, use_sparse_gamma: bool = True,
                              include_diagonal: bool = True, complex_mul_flops: int = 6,
                              complex_add_flops: int = 2, real_complex_mul_flops: int = 2) -> int:
        """Flops of one D application over the lattice and batch (wilson.py:417-437)."""
        per = self.flops_per_site_matvec(nc, use_sparse_gamma, include_diagonal, complex_mul_flops,
                                         complex_add_flops, real_complex_mul_flops)
        return int(per * int(volume) * int(batch))
