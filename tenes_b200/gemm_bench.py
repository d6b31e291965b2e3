"""Microbenchmark of the library's contraction kernels through tg_bench_gemm:

    python -m tenes_b200.gemm_bench M N K [layout] [prec] [iters]

layout 0: A row-major (M, K), B row-major (K, N); 1: B column-major (the rSVD
panel products).  prec 0: FP64 DMMA; 1: 3xTF32 on tcgen05.  Prints the average
device time of one product and its algorithmic rate (2 M N K flop)."""

import ctypes as C
import sys

from . import _lib


def main(argv=None) -> int:
    a = [int(x) for x in (sys.argv[1:] if argv is None else argv)]
    if len(a) < 3:
        print(__doc__)
        return 1
    M, N, K = a[:3]
    layout = a[3] if len(a) > 3 else 0
    prec = a[4] if len(a) > 4 else 0
    iters = a[5] if len(a) > 5 else 10
    lib = _lib.load()
    ms = C.c_double()
    _lib.check(lib.tg_bench_gemm(M, N, K, layout, prec, iters, C.byref(ms)))
    tf = 2.0 * M * N * K / (ms.value * 1e-3) / 1e12
    print(f"M={M} N={N} K={K} layout={layout} prec={prec}: {ms.value * 1e3:.1f} us  {tf:.1f} TFLOP/s", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
