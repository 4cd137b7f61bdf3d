"""Loader for the native extension (``_C``) over ``libdreamplace_b200.so``.

There is no fallback: every op in this package runs its CUDA kernels through
this module, and importing it without the built extension raises with the
build command to run.
"""
import os

_here = os.path.dirname(os.path.abspath(__file__))

try:
    import torch  # noqa: F401  (loads libtorch / libc10 before the extension)
    from . import _C as C  # noqa: N812
except ImportError as e:  # pragma: no cover - exercised only on unbuilt trees
    raise ImportError(
        "dreamplace_b200 native extension is not built (%s); run "
        "`python -m dreamplace_b200.build` (needs nvcc for sm_100a)" % e) from e

PREC = {"fp32": 0, "tf32": 1, "bf16": 2, "split_bf16": 3}


def precision_code(p):
    if isinstance(p, int):
        if p not in PREC.values():
            raise ValueError("unknown DCT precision %r" % p)
        return p
    try:
        return PREC[str(p).lower()]
    except KeyError:
        raise ValueError("unknown DCT precision %r (expected one of %s)" % (p, sorted(PREC))) from None


def require_cuda(t, name="tensor"):
    if not t.is_cuda:
        raise RuntimeError("dreamplace_b200 runs on CUDA only: %s is on %s" % (name, t.device))
