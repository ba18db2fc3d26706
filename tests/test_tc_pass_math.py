"""CPU checks of the arithmetic identities the tensor-core rounding pass relies
on, restated in exact rational arithmetic (no GPU).

1. The risk-plane GEMM (gemm_tc.cu, gemm3m_lead_path_kernel) sums the risk
   integral of MergeProductsWithPath (cgemm_compute_kernel.cpp:432-474),
   sum_k w_k (s_{k-1}^2 + s_{k-1} s_k + s_k^2) with s_0 = 0, by parts:
   acc = sum_{k<K} s_k (2 s_k + s_{k-1}) over the full segments, then
   w (acc - s_{K-1}^2) + w_K (s_{K-1}^2 + s_{K-1} s_K + s_K^2).
2. The exact recompute (ozaki.cu) reconstructs x = sum_m y_m w_m - k M with
   w_m = u_m (M / p_m) mod M, u_m = (M / p_m)^-1 mod p_m, three 40-bit FP64
   limbs and k = rint(s2 rn(2^80 / M) + s1 rn(2^40 / M)).
"""
import math
import random
from fractions import Fraction

MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199]
BETA = 47
MAX_N = 4096


def test_risk_integral_by_parts_is_the_segment_integral():
    rng = random.Random(5)
    for _ in range(2000):
        segments = rng.randint(1, 40)
        d = rng.choice([32, 64, 128])
        last = rng.randint(1, d)
        s = [Fraction(0)] + [Fraction(rng.randint(-10**6, 10**6), rng.randint(1, 1000)) for _ in range(segments)]
        w = [Fraction(d, 9)] * (segments - 1) + [Fraction(last, 9)]
        direct = sum(w[k - 1] * (s[k - 1] ** 2 + s[k - 1] * s[k] + s[k] ** 2) for k in range(1, segments + 1))
        acc = sum(s[k] * (2 * s[k] + s[k - 1]) for k in range(1, segments))
        K = segments
        by_parts = Fraction(d, 9) * (acc - s[K - 1] ** 2) + w[K - 1] * (s[K - 1] ** 2 + s[K - 1] * s[K] + s[K] ** 2)
        assert by_parts == direct


def _crt():
    M = math.prod(MODULI)
    ws = []
    for p in MODULI:
        W = M // p
        u = pow(W % p, -1, p)
        ws.append((W * u) % M)
    return M, ws


def test_moduli_and_reconstruction_constants():
    M, ws = _crt()
    for i, p in enumerate(MODULI):
        for j, q in enumerate(MODULI):
            if i < j:
                assert math.gcd(p, q) == 1
    for w, p in zip(ws, MODULI):
        assert w % p == 1
        assert all(w % q == 0 for q in MODULI if q != p)
    # every exact product of order <= 4096 lies within M / 8
    assert 2 * MAX_N * 2 ** (2 * BETA) <= M // 8


def test_limb_reconstruction_with_k_from_the_limb_sums():
    M, ws = _crt()
    mask = (1 << 40) - 1
    limbs = [[float((w >> (40 * l)) & mask) for l in range(3)] for w in ws]
    m_limbs = [float((M >> (40 * l)) & mask) for l in range(3)]
    k2, k1 = float(Fraction(2 ** 80, M)), float(Fraction(2 ** 40, M))
    rng = random.Random(7)
    bound = 2 * MAX_N * 2 ** (2 * BETA)
    for _ in range(5000):
        x = rng.choice([0, 1, -1, rng.randint(-bound, bound), rng.randint(-2 ** 30, 2 ** 30)])
        y = [x % p for p in MODULI]
        s = [0.0, 0.0, 0.0]
        for ym, wl in zip(y, limbs):
            for l in range(3):
                s[l] = s[l] + ym * wl[l]
                assert s[l] < 2.0 ** 52  # every product and partial sum exact
        S = int(s[2]) * 2 ** 80 + int(s[1]) * 2 ** 40 + int(s[0])
        est = s[2] * k2 + s[1] * k1
        assert abs(est - float(Fraction(S, M))) < 2.0 ** -30
        k = round(est)
        assert S - k * M == x
        d = [s[l] - k * m_limbs[l] for l in range(3)]
        assert all(float(int(v)) == v and abs(v) < 2.0 ** 53 for v in d)
        got = (d[2] * 2.0 ** 40 + d[1]) * 2.0 ** 40 + d[0]
        assert abs(got - x) <= abs(x) * 2.0 ** -52
