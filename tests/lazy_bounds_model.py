"""Interval model of the lazy GF(M61) arithmetic in montmul_b200/csrc (mm_field.cuh, mm_ntt.cuh,
mm_kernels.cuh): every operation of the radix-8/4/2 DIF and DIT butterflies, the Karatsuba
twiddle product, the squaring, the constant products and the wraparound half-pointwise step,
as maximum values. It checks that no intermediate passes 2^64, that each offset K p of a
subtraction covers the subtrahend, and that every value stored between passes is below
2^61 + 2^34. tests/test_lazy_bounds.py runs it.
"""
P = (1 << 61) - 1
TOP = (1 << 64) - 1
class V:
    def __init__(s, m): assert 0 <= m <= TOP, hex(m); s.m = m
def add(a, b): return V(a.m + b.m)
def sub(a, b, K): assert K * P >= b.m, (K, hex(b.m)); return V(a.m + K * P)
def fold(x): return V(P + (x.m >> 61))
def rot(x): return V(P + (x.m >> 31))
def mul1(a, b):  # (P & p) + (P >> 61), product < 2^125
    prod = a.m * b.m; assert prod < 1 << 125; return V(P + (prod >> 61))
class C:
    def __init__(s, re, im): s.re, s.im = re, im
def cadd(a, b): return C(add(a.re, b.re), add(a.im, b.im))
def csub(a, b, K): return C(sub(a.re, b.re, K), sub(a.im, b.im, K))
def csub_i(a, b, K): return C(sub(b.im, a.im, K), sub(a.re, b.re, K))      # (a - b) i
def cadd_mi(u, v, K): return C(add(u.re, v.im), sub(u.im, v.re, K))        # u + (-i) v
def csub_mi(u, v, K): return C(sub(u.re, v.im, K), add(u.im, v.re))        # u - (-i) v
def w8(x, K): return C(rot(sub(x.re, x.im, K)), rot(add(x.re, x.im)))      # x (1+i) 2^30
def v8(x, K): return C(rot(add(x.re, x.im)), rot(sub(x.im, x.re, K)))      # x (1-i) 2^30
def mi(x, K): return C(x.im, sub(V(0), x.re, K))                           # x (-i)
def cfold(x): return C(fold(x.re), fold(x.im))
W = V(P - 1)  # canonical constant
def kmul(x):  # Karatsuba with canonical (wr, wr+wi, wi-wr); x components <= ONE
    k1 = mul1(add(x.re, x.im), W); k2 = mul1(x.re, W); k3 = mul1(x.im, W)
    return C(fold(sub(k1, k3, 3)), fold(add(k1, k2)))
ONE = (1 << 61) + (1 << 34)
def inp(): return C(V(ONE), V(ONE))
def check_one(c, what):
    assert c.re.m <= ONE and c.im.m <= ONE, (what, hex(c.re.m), hex(c.im.m))

def dif8(tw):
    x = [inp() for _ in range(8)]
    a = [cfold(cadd(x[k], x[k + 4])) for k in range(4)]
    b = [cfold(csub(x[0], x[4], 2)), w8(csub(x[1], x[5], 2), 4), cfold(csub_i(x[2], x[6], 2)), w8(csub_i(x[3], x[7], 2), 4)]
    c0, c2, c1, c3 = cadd(a[0], a[2]), csub(a[0], a[2], 2), cadd(a[1], a[3]), csub_i(a[1], a[3], 2)
    d0, d2, d1, d3 = cadd(b[0], b[2]), csub(b[0], b[2], 2), cadd(b[1], b[3]), csub_i(b[1], b[3], 2)
    y = [cadd(c0, c1), csub(c0, c1, 3), cadd(c2, c3), csub(c2, c3, 4), cadd(d0, d1), csub(d0, d1, 3), cadd(d2, d3), csub(d2, d3, 4)]
    out = [cfold(y[0])] + [kmul(cfold(y[k])) if tw else cfold(y[k]) for k in range(1, 8)]
    for k, o in enumerate(out): check_one(o, f"dif8 out {k}")
    return y

def dit8(tw):
    x = [kmul(inp()) if (tw and k) else inp() for k in range(8)]
    c = []
    for k in range(0, 8, 2):
        c += [cfold(cadd(x[k], x[k + 1])), cfold(csub(x[k], x[k + 1], 2))]
    a0, a2 = cadd(c[0], c[2]), csub(c[0], c[2], 2)
    a1, a3 = cadd_mi(c[1], c[3], 2), csub_mi(c[1], c[3], 2)
    b0, b2 = cadd(c[4], c[6]), csub(c[4], c[6], 2)
    b1, b3 = cadd_mi(c[5], c[7], 2), csub_mi(c[5], c[7], 2)
    v1 = v8(b1, 4)
    v3 = v8(mi(b3, 4), 4)
    y = [None] * 8
    y[0], y[4] = cadd(a0, b0), csub(a0, b0, 3)
    y[1], y[5] = cadd(a1, v1), csub(a1, v1, 2)
    y[2] = C(add(a2.re, b2.im), sub(a2.im, b2.re, 4))     # a2 + (-i) b2
    y[6] = C(sub(a2.re, b2.im, 4), add(a2.im, b2.re))     # a2 - (-i) b2
    y[3], y[7] = cadd(a3, v3), csub(a3, v3, 2)
    out = [cfold(v) for v in y]
    for k, o in enumerate(out): check_one(o, f"dit8 out {k}")
    return y

def dif4(tw):
    x = [inp() for _ in range(4)]
    a0, b0 = cadd(x[0], x[2]), csub(x[0], x[2], 2)
    a1, b1 = cadd(x[1], x[3]), csub_i(x[1], x[3], 2)
    y = [cadd(a0, a1), csub(a0, a1, 3), cadd(b0, b1), csub(b0, b1, 4)]
    out = [cfold(y[0])] + [kmul(cfold(y[k])) if tw else cfold(y[k]) for k in range(1, 4)]
    for k, o in enumerate(out): check_one(o, f"dif4 out {k}")

def dit4(tw):
    x = [kmul(inp()) if (tw and k) else inp() for k in range(4)]
    c0, c1, c2, c3 = cadd(x[0], x[1]), csub(x[0], x[1], 2), cadd(x[2], x[3]), csub(x[2], x[3], 2)
    y = [cadd(c0, c2), cadd_mi(c1, c3, 4), csub(c0, c2, 3), csub_mi(c1, c3, 4)]
    out = [cfold(v) for v in y]
    for k, o in enumerate(out): check_one(o, f"dit4 out {k}")

def dif2(tw):
    x = [inp(), inp()]
    y = [cadd(x[0], x[1]), csub(x[0], x[1], 2)]
    out = [cfold(y[0]), kmul(cfold(y[1])) if tw else cfold(y[1])]
    for o in out: check_one(o, "dif2")

def check_butterflies():
    for tw in (False, True):
        dif8(tw); dit8(tw); dif4(tw); dit4(tw); dif2(tw)

# ---- pointwise operations ----
def kmul_lazy_sums(x):
    """lkmulc: constants (wr, wi) canonical, s = wr + wi and d = wi - wr + p formed lazily."""
    s = add(W, W); d = sub(W, W, 1)
    k1 = mul1(add(x.re, x.im), W); k2 = mul1(x.re, d); k3 = mul1(x.im, s)
    return C(fold(sub(k1, k3, 4)), fold(add(k1, k2)))


def check_pointwise():
    # lsqr_scale with c = 4
    x = inp()
    re = fold(mul1(add(x.re, x.im), sub(x.re, x.im, 2)))
    t = mul1(x.re, x.im)
    im = fold(add(t, t))
    check_one(C(fold(V(re.m * 4)), fold(V(im.m * 4))), "square")
    # lreal_times: a 32-bit limb times a canonical constant
    check_one(C(fold(mul1(V((1 << 32) - 1), W)), fold(mul1(V((1 << 32) - 1), W))), "weighted input")
    check_one(kmul_lazy_sums(inp()), "kmul lazy sums")
    # half_pointwise: e = zp + conj zq, d = zp - conj zq, out = e A + d B
    zp, zq = inp(), inp()
    e = C(add(zp.re, zq.re), add(zp.im, sub(V(0), zq.im, 2)))
    d = C(sub(zp.re, zq.re, 2), add(zp.im, zq.im))
    check_one(cfold(cadd(kmul_lazy_sums(cfold(e)), kmul_lazy_sums(cfold(d)))), "half pointwise")
    # lkmul_re: re(x c) = x.re c.re + x.im (p - c.im)
    check_one(C(fold(add(mul1(V(ONE), W), mul1(V(ONE), W))), V(0)), "real only")
