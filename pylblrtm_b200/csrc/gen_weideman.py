"""Generate weideman_coeffs.h: coefficients of Weideman's rational approximation.

J.A.C. Weideman (1994), "Computation of the complex error function", SIAM J.
Numer. Anal. 31(5):1497-1518: for Im z >= 0,

    w(z) ~ 2 sum_{n=1..N} a_n Z^(n-1) / (L - iz)^2 + 1 / (sqrt(pi) (L - iz)),
    Z = (L + iz) / (L - iz),  L = (N / sqrt(2))^(1/2),

where a_n are the Fourier coefficients of (L^2 + t^2) exp(-t^2) under the map
t = L tan(theta/2), obtained here by an FFT on 4N points. Two sets: N = 36 (|w|
relative error <= 2e-14 for |z| <= 6; the float64 engine) and
N = 28 (the near zones of the float32 multi-level engine and its Jacobians: Re w relative error <= 7e-7
for y >= 1e-4 and <= 1e-8 for y >= 0.01 inside |z|^2 < 36, against
scipy.special.wofz; float32 rounding of the sums is ~1e-7). Run:

    python pylblrtm_b200/csrc/gen_weideman.py > pylblrtm_b200/csrc/weideman_coeffs.h
"""

import numpy as np

SETS = (("LBL_WEIDEMAN", 36), ("LBL_WEIDEMAN28", 28))


def coefficients(n: int):
    m = 2 * n
    k = np.arange(-m + 1, m)
    big_l = np.sqrt(n / np.sqrt(2.0))
    t = big_l * np.tan(k * np.pi / m / 2.0)
    f = np.concatenate([[0.0], np.exp(-t ** 2) * (big_l ** 2 + t ** 2)])
    a = np.real(np.fft.fft(np.fft.fftshift(f))) / (2 * m)
    return big_l, a[1:n + 1]          # a_1 .. a_N


def main():
    print("// Generated by gen_weideman.py: Weideman (1994) rational approximation of w(z).")
    print("#pragma once")
    for name, n in SETS:
        big_l, a = coefficients(n)
        print(f"#define {name}_N {n}")
        print(f"#define {name}_L {float(big_l)!r}")
        print("// a_1 .. a_N (polynomial in Z: sum a_n Z^(n-1)), as an initializer list")
        print(f"#define {name}_COEFFS \\")
        for i in range(0, n, 3):
            tail = ", \\" if i + 3 < n else ""
            print("    " + ", ".join(repr(float(v)) for v in a[i:i + 3]) + tail)


if __name__ == "__main__":
    main()
