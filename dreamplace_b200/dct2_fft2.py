"""2-D DCT family of the Poisson solve, as GEMMs on the tensor cores.

Drop-in for the reference's ``dreamplace/ops/dct/dct2_fft2.py``: modules
``DCT2``, ``IDCT2``, ``IDCT_IDXST``, ``IDXST_IDCT`` taking ``(expkM, expkN)`` and
transforming an ``M x N`` map with ``.forward(x)``.  The reference computes them
with a real FFT and twiddle kernels (dct/src/dct2_fft2_cuda_kernel.cu); here each
2-D transform is two dense products with cosine / sine matrices,

    dct2_fft2(x)   = 4/(M N) * C_M  x C_N^T      C_n[k,i] = cos(pi (2i+1) k / (2n))
    idct2_fft2(y)  = 4 * Ch_M y Ch_N^T          Ch_n[u,p] = w_p cos(pi p (u+1/2) / n),  w_0 = 1/2
    idct_idxst(y)  = 4 * Ch_M y Sh_N^T          Sh_n[u,p] = sin(pi p (u+1/2) / n)
    idxst_idct(y)  = 4 * Sh_M y Ch_N^T

(identities checked against the reference CPU op ``dct2_fft2_cpp`` to 2e-14 in
fp64).  ``precision`` picks the arithmetic: ``fp32`` (SIMT, the plain form),
``tf32``, ``bf16`` or ``split_bf16`` (hi*hi + hi*lo + lo*hi, fp32 accumulation).
The matrices are built in fp64 and rounded once.
"""

import numpy as np
import torch
from torch import nn

from ._native import C, precision_code, require_cuda

EPI_STORE, EPI_STORE_T, EPI_SPECTRAL, EPI_ENERGY = 0, 1, 2, 3


def get_exact_expk(N, dtype, device):
    """exp(-j pi u / (2N)) as [N, 2] (cos, -sin); reference
    dreamplace/ops/dct/discrete_spectral_transform.py:63-69.  Kept for API
    compatibility: the GEMM transforms do not read it."""
    u = torch.arange(N, dtype=dtype, device=device).mul_(np.pi / (2 * N))
    return torch.stack([u.cos(), -u.sin()], dim=-1).contiguous()


precompute_expk = get_exact_expk


def cos_matrix(n):
    """C_n[k, i] = cos(pi (2i+1) k / (2n)), fp64."""
    k = np.arange(n, dtype=np.float64)[:, None]
    i = np.arange(n, dtype=np.float64)[None, :]
    return np.cos(np.pi * (2 * i + 1) * k / (2 * n))


def icos_matrix(n):
    """Ch_n[u, p] = w_p cos(pi p (u + 1/2) / n), w_0 = 1/2, fp64."""
    u = np.arange(n, dtype=np.float64)[:, None]
    p = np.arange(n, dtype=np.float64)[None, :]
    m = np.cos(np.pi * p * (u + 0.5) / n)
    m[:, 0] *= 0.5
    return m


def isin_matrix(n):
    """Sh_n[u, p] = sin(pi p (u + 1/2) / n), fp64."""
    u = np.arange(n, dtype=np.float64)[:, None]
    p = np.arange(n, dtype=np.float64)[None, :]
    return np.sin(np.pi * p * (u + 0.5) / n)


class Operand:
    """A GEMM operand in the storage format of a precision: fp32, bf16 hi, or bf16 hi+lo."""

    def __init__(self, shape, prec, device):
        self.prec = prec
        if prec in (0, 1):
            self.f32 = torch.empty(shape, dtype=torch.float32, device=device)
            self.hi = self.lo = None
        else:
            self.f32 = None
            self.hi = torch.empty(shape, dtype=torch.bfloat16, device=device)
            self.lo = torch.empty(shape, dtype=torch.bfloat16, device=device) if prec == 3 else None

    @classmethod
    def from_fp64(cls, m, prec, device):
        op = cls(m.shape, prec, device)
        if prec in (0, 1):
            op.f32.copy_(torch.from_numpy(m.astype(np.float32)))
        else:
            t64 = torch.from_numpy(m)
            hi = t64.to(torch.bfloat16)
            op.hi.copy_(hi)
            if op.lo is not None:
                op.lo.copy_((t64 - hi.to(torch.float64)).to(torch.bfloat16))
        return op

    @classmethod
    def from_tensor(cls, x, prec, scale=1.0):
        return cls(tuple(x.shape), prec, x.device).fill(x, scale)

    def fill(self, x, scale=1.0):
        """Stores scale * x (fp32, this operand's shape) in this operand's format."""
        C.prepare_operand(self.prec, x.contiguous(), float(scale), self.f32, self.hi, self.lo)
        return self

    @property
    def main(self):
        return self.f32 if self.f32 is not None else self.hi

    def as_a(self, d):
        d["a_hi"], d["a_lo"] = self.main, self.lo
        return d

    def as_b(self, d):
        d["b_hi"], d["b_lo"] = self.main, self.lo
        return d

    def as_out_t(self, d):
        if self.f32 is not None:
            d["out_f32"] = self.f32
        else:
            d["out_hi"], d["out_lo"] = self.hi, self.lo
        return d


_MATRIX_CACHE = {}


def transform_matrices(n, prec, device):
    """(C_n, Ch_n, Sh_n) as operands of ``prec`` on ``device`` (cached)."""
    key = (n, prec, str(device))
    if key not in _MATRIX_CACHE:
        _MATRIX_CACHE[key] = tuple(Operand.from_fp64(f(n), prec, device)
                                   for f in (cos_matrix, icos_matrix, isin_matrix))
    return _MATRIX_CACHE[key]


def transform_2d(x, left, right, alpha, prec, out=None):
    """out = alpha * left @ x @ right^T via two GEMMs (x: M x N fp32)."""
    M, N = x.shape
    a = Operand.from_tensor(x, prec) if prec != 0 else None
    t = Operand((N, M), prec, x.device)
    g1 = dict(lda=N, ldb=N, epilogue=EPI_STORE_T, alpha=1.0, ldc=M)
    if a is None:
        g1["a_hi"] = x.contiguous()
    else:
        a.as_a(g1)
    right.as_b(g1)
    t.as_out_t(g1)
    C.transform_gemm(prec, M, N, N, [g1])
    if out is None:
        out = torch.empty(M, N, dtype=torch.float32, device=x.device)
    g2 = dict(lda=M, ldb=M, epilogue=EPI_STORE, alpha=float(alpha), ldc=N, out_f32=out)
    left.as_a(g2)
    t.as_b(g2)
    C.transform_gemm(prec, M, N, M, [g2])
    return out


class _Transform(nn.Module):
    kind = None

    def __init__(self, expkM=None, expkN=None, precision="fp32"):
        super().__init__()
        self.expkM = expkM
        self.expkN = expkN
        self.precision = precision_code(precision)
        self.out = None

    def forward(self, x):
        require_cuda(x, "x")
        if x.dtype != torch.float32:
            raise TypeError("dreamplace_b200 transforms take float32 maps, got %s" % x.dtype)
        M, N = x.size(-2), x.size(-1)
        cM, chM, shM = transform_matrices(M, self.precision, x.device)
        cN, chN, shN = transform_matrices(N, self.precision, x.device)
        left, right, alpha = {
            "dct2": (cM, cN, 4.0 / (M * N)),
            "idct2": (chM, chN, 4.0),
            "idct_idxst": (chM, shN, 4.0),
            "idxst_idct": (shM, chN, 4.0),
        }[self.kind]
        if self.out is None or self.out.shape != (M, N) or self.out.device != x.device:
            self.out = torch.empty(M, N, dtype=torch.float32, device=x.device)
        return transform_2d(x.reshape(M, N), left, right, alpha, self.precision, self.out)


class DCT2(_Transform):
    """dct2_fft2: 4/(MN) C_M x C_N^T (reference dct/dct2_fft2.py:DCT2)."""
    kind = "dct2"


class IDCT2(_Transform):
    """idct2_fft2: 4 Ch_M y Ch_N^T (reference dct/dct2_fft2.py:IDCT2)."""
    kind = "idct2"


class IDCT_IDXST(_Transform):  # noqa: N801 (reference name)
    """idct_idxst: 4 Ch_M y Sh_N^T (reference dct/dct2_fft2.py:IDCT_IDXST)."""
    kind = "idct_idxst"


class IDXST_IDCT(_Transform):  # noqa: N801 (reference name)
    """idxst_idct: 4 Sh_M y Ch_N^T (reference dct/dct2_fft2.py:IDXST_IDCT)."""
    kind = "idxst_idct"


def gemm_flops(M, N, prec, transforms):
    """Algorithmic flops of ``transforms`` 2-D transforms at M x N (2 GEMMs each)."""
    k = 3 if prec == 3 else 1
    return transforms * k * 2.0 * M * N * (M + N)
