"""Generate weideman_coeffs.h: coefficients of Weideman's rational approximation.

J.A.C. Weideman (1994), "Computation of the complex error function", SIAM J.
Numer. Anal. 31(5):1497-1518: for Im z >= 0,

    w(z) ~ 2 sum_{n=1..N} a_n Z^(n-1) / (L - iz)^2 + 1 / (sqrt(pi) (L - iz)),
    Z = (L + iz) / (L - iz),  L = (N / sqrt(2))^(1/2),

where a_n are the Fourier coefficients of (L^2 + t^2) exp(-t^2) under the map
t = L tan(theta/2), obtained here by an FFT on 4N points. Run:

    python pylblrtm_b200/csrc/gen_weideman.py > pylblrtm_b200/csrc/weideman_coeffs.h
"""

import numpy as np

N = 36


def coefficients(n: int):
    m = 2 * n
    k = np.arange(-m + 1, m)
    big_l = np.sqrt(n / np.sqrt(2.0))
    t = big_l * np.tan(k * np.pi / m / 2.0)
    f = np.concatenate([[0.0], np.exp(-t ** 2) * (big_l ** 2 + t ** 2)])
    a = np.real(np.fft.fft(np.fft.fftshift(f))) / (2 * m)
    return big_l, a[1:n + 1]          # a_1 .. a_N


def main():
    big_l, a = coefficients(N)
    print("// Generated by gen_weideman.py: Weideman (1994) rational approximation of w(z).")
    print("#pragma once")
    print(f"#define LBL_WEIDEMAN_N {N}")
    print(f"#define LBL_WEIDEMAN_L {float(big_l)!r}")
    print("// a_1 .. a_N (polynomial in Z: sum a_n Z^(n-1)), as an initializer list")
    print("#define LBL_WEIDEMAN_COEFFS \\")
    for i in range(0, N, 3):
        tail = ", \\" if i + 3 < N else ""
        print("    " + ", ".join(repr(float(v)) for v in a[i:i + 3]) + tail)


if __name__ == "__main__":
    main()
