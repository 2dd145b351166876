// Host-side table builders of the CUDA library, checked without a GPU:
//  * pxp::adi_const_staged_tables -- the ADI one-wave kernel's staged
//    Thomas-factor tables and the run of chunks whose entries are bit for bit
//    equal (the kernel reads the run's first chunk for every chunk in it);
//  * pxp::fft3d_lines_tw_exponents -- the exponents of the FFTSolver3D line
//    kernel's twiddle table.
// Prints one line per check and exits non-zero on the first failure.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <vector>

namespace pxp {
bool adi_const_staged_tables(int n, const double *g, const double *h, double *out, int run[2]);
int fft3d_lines_tw_exponents(int n, int *out, int cap);
}  // namespace pxp

using cd = std::complex<double>;

static int fail(const char *what) {
  std::printf("FAIL %s\n", what);
  return 1;
}

// Thomas factors of the vacuum ADI matrix (diagonal 1/dz + i/(k dx^2),
// off-diagonal -0.5 i/(k dx^2)) padded to nw rows, as the solver builds them.
static void factors(int n, int nw, double dz, std::vector<cd> &pad) {
  const double k = 2.0 * std::acos(-1.0) / 0.1, dx = 1000.0 / (n - 1);
  const cd im(0.0, 1.0);
  const cd diag = 1.0 / dz + im / (k * dx * dx), sub = -0.5 * im / (k * dx * dx);
  std::vector<cd> g(n), h(n);
  cd den = diag;
  for (int i = 0; i < n; ++i) {
    if (i > 0) den = diag - sub * (sub * g[i - 1]);
    g[i] = cd(1.0) / den;
    h[i] = -sub * g[i];
  }
  pad.assign(2 * (size_t)nw, cd(0.0));
  for (int i = 0; i < nw; ++i) {
    pad[i] = i < n ? g[i] : cd(1.0, 0.0);
    pad[nw + i] = i < n ? h[i] : cd(0.0, 0.0);
  }
}

static int check_adi(int n, int nw, double dz, int want_c0, int want_c1) {
  std::vector<cd> pad, out(4 * (size_t)nw);
  factors(n, nw, dz, pad);
  int run[2] = {-1, -1};
  const double *t = reinterpret_cast<const double *>(pad.data());
  if (!pxp::adi_const_staged_tables(nw, t, t + 2 * nw, reinterpret_cast<double *>(out.data()), run))
    return fail("adi_const_staged_tables refused a one-wave length");
  std::printf("adi n=%d nw=%d run=[%d,%d)\n", n, nw, run[0], run[1]);
  if (want_c0 >= 0 && (run[0] != want_c0 || run[1] != want_c1)) return fail("adi run bounds");
  // every chunk of the run holds, in all four tables, its first chunk's bits
  const int M = 8, P = nw / M;
  auto slot = [&](int c, int m) { return m * P + (c ^ (m & 7)); };
  for (int c = run[0] + 1; c < run[1]; ++c)
    for (int tb = 0; tb < 4; ++tb)
      for (int m = 0; m < M; ++m)
        if (std::memcmp(&out[(size_t)tb * nw + slot(c, m)], &out[(size_t)tb * nw + slot(run[0], m)],
                        sizeof(cd)) != 0)
          return fail("chunk of the run differs from its first chunk");
  // and the run is maximal at its ends
  auto same = [&](int a, int b) {
    for (int tb = 0; tb < 4; ++tb)
      for (int m = 0; m < M; ++m)
        if (std::memcmp(&out[(size_t)tb * nw + slot(a, m)], &out[(size_t)tb * nw + slot(b, m)],
                        sizeof(cd)) != 0)
          return false;
    return true;
  };
  if (run[1] > run[0]) {
    if (run[0] > 0 && same(run[0] - 1, run[0])) return fail("run could start earlier");
    if (run[1] < P && same(run[1], run[0])) return fail("run could end later");
  }
  return 0;
}

static int check_tw(int n, int want) {
  std::vector<int> ex(n);
  const int cnt = pxp::fft3d_lines_tw_exponents(n, ex.data(), n);
  std::printf("tw n=%d entries=%d\n", n, cnt);
  if (cnt != want) return fail("twiddle table length");
  if (cnt == 0) return 0;
  // radix-8 passes before the last, each 7 * NS entries (r - 1) * NS + k with
  // exponent r * k * n / (8 NS); the first pass's NS is the first-pass radix
  int lg = 0;
  while ((1 << lg) < n) ++lg;
  const int r0 = lg % 3 == 0 ? 8 : (lg % 3 == 1 ? 2 : 4);
  int i = 0;
  for (int ns = r0; i < cnt; ns *= 8)
    for (int e = 0; e < 7 * ns; ++e, ++i) {
      const int r = e / ns + 1, kk = e % ns;
      if (ex[i] != r * kk * (n / (8 * ns))) return fail("twiddle exponent");
    }
  return 0;
}

int main() {
  // the benchmark's ADI grid (1024 nodes on [-500, 500], dz/2 = 500): the
  // factors reach their limit after 51 rows, so chunks 7..127 coincide
  if (check_adi(1024, 1024, 500.0, 7, 128)) return 1;
  // padded grids: the padding chunks (rows n .. nw-1) end the run
  if (check_adi(1000, 1024, 500.0, 7, 125)) return 1;
  if (check_adi(700, 768, 500.0, 5, 87)) return 1;
  // a strongly diagonal matrix (short dz): any run found must still hold
  if (check_adi(512, 512, 5.0, -1, -1)) return 1;
  if (check_tw(4096, 7 * 8 + 7 * 64)) return 1;
  if (check_tw(2048, 7 * 4 + 7 * 32)) return 1;
  if (check_tw(1024, 7 * 2 + 7 * 16)) return 1;
  if (check_tw(512, 0)) return 1;
  std::printf("OK\n");
  return 0;
}
