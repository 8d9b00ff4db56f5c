"""Generate tests/golden/kiss_fft.npz: input/output vectors of the reference's own
KISS FFT (fftMPI's kissfft.h, double precision, src/fftmpi/src/kissfft.h with
src/fftmpi/src/ffttype.h), which oracle/build_ref.sh compiles from the reference tree
into oracle/_ref/libkissref.so.

The fixtures pin the oracle's DFT (the stand-in for FFTW 3.3.8, a dependency the
reference tree does not vendor) on machines where the reference tree is absent.

Contents (all float64; complex values stored as separate re/im arrays):
  1-D: for each n in N1D, a seeded dyadic-rational input x_n and the KISS forward (sign -1) and
       backward (sign +1, unnormalised) transforms;
  2-D: for each (ny, nx) in N2D, a seeded input and its forward/backward 2-D
       transform, composed from KISS 1-D transforms of every row (length nx) and then
       every column (length ny): the same separable c2c DFT that
       fftw_plan_dft_2d computes (src/PRESSURE/fft_interface.f90:580-591,626-637).

Run:  bash oracle/build_ref.sh && python tests/golden/make_kiss_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

# lengths with radix 2/3/4/5 factors, generic (prime) factors, and the pressure
# solver's typical horizontal sizes (maxx - 5 interior points of padded grids)
N1D = [1, 2, 3, 4, 5, 7, 8, 9, 12, 15, 16, 25, 27, 30, 45, 49, 59, 60, 64, 96, 121, 125, 128, 160, 243, 256]
N2D = [(8, 12), (12, 20), (30, 18), (5, 7), (9, 1), (27, 16), (16, 32)]
SEED = 20250601


def dyadic(rng, shape) -> np.ndarray:
    """Seeded complex input with dyadic-rational parts k/1024, |k| <= 4096: exact in any
    format, and small in the compressed fixture."""
    return (rng.integers(-4096, 4097, shape) + 1j * rng.integers(-4096, 4097, shape)) / 1024.0


def kiss2d(x: np.ndarray, inverse: bool) -> np.ndarray:
    ny, nx = x.shape
    rows = np.stack([O.kiss_fft(x[m], inverse=inverse) for m in range(ny)])
    return np.stack([O.kiss_fft(rows[:, l], inverse=inverse) for l in range(nx)], axis=1)


def main() -> None:
    if O.kiss_ref() is None:
        sys.exit("oracle/_ref/libkissref.so is missing: run oracle/build_ref.sh (needs the reference tree)")
    rng = np.random.default_rng(SEED)
    out = {"n1d": np.array(N1D), "n2d": np.array(N2D)}
    for n in N1D:
        x = dyadic(rng, (n,))
        f, b = O.kiss_fft(x), O.kiss_fft(x, inverse=True)
        for name, v in (("x", x), ("fwd", f), ("bwd", b)):
            out[f"1d_{n}_{name}_re"], out[f"1d_{n}_{name}_im"] = v.real.copy(), v.imag.copy()
    for ny, nx in N2D:
        x = dyadic(rng, (ny, nx))
        f, b = kiss2d(x, False), kiss2d(x, True)
        for name, v in (("x", x), ("fwd", f), ("bwd", b)):
            out[f"2d_{ny}x{nx}_{name}_re"], out[f"2d_{ny}x{nx}_{name}_im"] = v.real.copy(), v.imag.copy()
    path = os.path.join(HERE, "kiss_fft.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
