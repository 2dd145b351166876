"""Why served mode holds its constant factors as split complex64 pairs.

A CPU restatement of the served-mode FFTSolver2D step (the device's Stockham
transform: a first pass of radix 2, 4 or 8, then radix-8 passes with the
dft8 of fft_smem.cuh) with every FP32 operation rounded as the device rounds
it, on the 2048-point waveguide of the benchmark's first configuration
shrunk to 512 points.  Three ways of holding the constant factors (table
twiddles, the 1/sqrt(2) inside dft8, the propagator and the transmission):

  * split: hi = fl32(w), lo = fl32(w - hi), product by the FMA chain of
    tw_mul(float2, float4) -- what the kernels do;
  * twiddles split but 1/sqrt(2) rounded to FP32;
  * every factor rounded to FP32, plain FP32 FMAs.

Against the FP64 step, the split form's relative intensity error stays at
the data-rounding level over 2000 steps, while a factor rounded to FP32
makes the error grow linearly with the step count (the field changes little
between steps, so the same rounding repeats).  FP32 FMAs are emulated in
FP64: a product of two FP32 values is exact there, and rounding the FP64 sum
to FP32 differs from a fused FP32 FMA only when the FP64 sum itself rounds,
which does not change these statistics."""
import numpy as np

F32, F64 = np.float32, np.float64


def _fma(a, b, c):
    return (a.astype(F64) * b.astype(F64) + c.astype(F64)).astype(F32)


def _split(v):
    hi = v.astype(F32)
    return hi, (v - hi.astype(F64)).astype(F32)


def _mul_split(x, y, wr, wi):
    """(x + iy)(wr + i wi) with split factors, the device's FMA chain."""
    hr, lr = _split(wr)
    hi, li = _split(wi)
    return (_fma(x, hr, _fma(-y, hi, _fma(x, lr, -(y * li)))),
            _fma(x, hi, _fma(y, hr, _fma(x, li, y * lr))))


def _mul_f32(x, y, wr, wi):
    wr, wi = wr.astype(F32), wi.astype(F32)
    return _fma(x, wr, -(y * wi)), _fma(x, wi, y * wr)


H = 0.70710678118654752440


def _half_split(a):
    hh = F32(H)
    hl = F32(H - float(hh))
    return _fma(a, np.full_like(a, hh), a * hl)


def _half_f32(a):
    return a * F32(H)


def _dft(v, sign, half):
    add = lambda p, q: (p[0] + q[0], p[1] + q[1])
    sub = lambda p, q: (p[0] - q[0], p[1] - q[1])
    muli = (lambda p: (p[1], -p[0])) if sign < 0 else (lambda p: (-p[1], p[0]))

    def d4(v0, v1, v2, v3):
        a0, a1, a2, a3 = add(v0, v2), sub(v0, v2), add(v1, v3), muli(sub(v1, v3))
        return add(a0, a2), add(a1, a3), sub(a0, a2), sub(a1, a3)

    if len(v) == 2:
        return [add(v[0], v[1]), sub(v[0], v[1])]
    if len(v) == 4:
        return list(d4(*v))
    a = [add(v[i], v[i + 4]) for i in range(4)]
    b = [sub(v[i], v[i + 4]) for i in range(4)]
    b1, b2, b3 = b[1], b[2], b[3]
    if sign < 0:
        b1 = (half(b1[0] + b1[1]), half(b1[1] - b1[0]))
        b2 = (b2[1], -b2[0])
        b3 = (half(b3[1] - b3[0]), half(-(b3[0] + b3[1])))
    else:
        b1 = (half(b1[0] - b1[1]), half(b1[0] + b1[1]))
        b2 = (-b2[1], b2[0])
        b3 = (half(-(b3[0] + b3[1])), half(b3[0] - b3[1]))
    A, B = d4(*a), d4(b[0], b1, b2, b3)
    return [A[0], B[0], A[1], B[1], A[2], B[2], A[3], B[3]]


def _plan(n):
    log = int(np.log2(n))
    r0 = 8 if log % 3 == 0 else (2 if log % 3 == 1 else 4)
    passes, ns = [(r0, 1)], r0
    while ns < n:
        passes.append((8, ns))
        ns *= 8
    plan = []
    for r, ns in passes:
        j = np.arange(n // r)
        k = j % ns
        plan.append((r, ns, [j + q * (n // r) for q in range(r)],
                     [(j - k) * r + k + q * ns for q in range(r)],
                     [np.exp(-2j * np.pi * q * k / (ns * r)) for q in range(r)]))
    return plan


def _fft(re, im, plan, sign, mul, half):
    for r, ns, idx_in, idx_out, tw in plan:
        v = []
        for q in range(r):
            x, y = re[idx_in[q]], im[idx_in[q]]
            if ns > 1 and q > 0:
                w = tw[q] if sign < 0 else np.conj(tw[q])
                x, y = mul(x, y, w.real, w.imag)
            v.append((x, y))
        out = _dft(v, sign, half)
        re, im = np.empty_like(re), np.empty_like(im)
        for q in range(r):
            re[idx_out[q]], im[idx_out[q]] = out[q]
    return re, im


def _intensity_errors(mul, half, n=512, nsteps=2000, checks=(500, 1000, 2000)):
    x = -250.0 + 500.0 / (n - 1) * np.arange(n)
    k, dz = 2 * np.pi / 0.1, 1000.0
    d = np.minimum(np.arange(n), n - 1 - np.arange(n))
    delta = np.where((np.abs(x) <= 25) & (d >= 25), 0.0, 7.5e-6)
    beta = np.where(np.abs(x) <= 25, 0.0, 1e-7)
    beta = np.where(d < 25, 1e-7 + (1e-4 - 1e-7) * (25 - d) / 25.0, beta)
    t = np.exp(-k * (beta + 1j * delta) * dz) / n
    idx = np.arange(n)
    kx = 2 * np.pi * np.where(idx > n // 2, n - idx, idx) / (500.0 / (n - 1) * n)
    kern = np.exp(-1j * kx ** 2 * dz / (2 * k))
    u = np.exp(-x ** 2 / 15.0 ** 2).astype(np.complex128)
    re, im = u.real.astype(F32), u.imag.astype(F32)
    plan = _plan(n)
    errs = {}
    for s in range(1, nsteps + 1):
        u = np.fft.ifft(np.fft.fft(u) * kern) * n * t
        re, im = _fft(re, im, plan, -1, mul, half)
        re, im = mul(re, im, kern.real, kern.imag)
        re, im = _fft(re, im, plan, +1, mul, half)
        re, im = mul(re, im, t.real, t.imag)
        if s in checks:
            i64 = np.abs(u) ** 2
            i32 = re.astype(F64) ** 2 + im.astype(F64) ** 2
            errs[s] = np.linalg.norm(i32 - i64) / np.linalg.norm(i64)
    return errs


def test_split_constants_keep_the_error_flat():
    split = _intensity_errors(_mul_split, _half_split)
    half_rounded = _intensity_errors(_mul_split, _half_f32)
    rounded = _intensity_errors(_mul_f32, _half_f32)
    assert max(split.values()) < 5e-6
    # a factor rounded to FP32: linear growth, far above the split form
    for errs in (half_rounded, rounded):
        assert errs[2000] > 1.6 * errs[1000] > 2.5 * errs[500] > 0
        assert errs[2000] > 20 * split[2000]
