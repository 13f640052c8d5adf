// wirespace_host.cu -- host code (no kernels): the cubic-spline resampling of
// many complex signals between the propagation grid and the wire grid, the
// inner loop of Prop2QW / QW2Prop (qwoptics.py:673-812) for every wire of a
// Maxwell step at once.
//
// The spline is the reference's rescale_1D_dpc (spliner.py:153-188) with the
// Forsythe-Malcolm-Moler spline of spline_dpc / seval_dpc
// (spliner.py:1287-1396): end conditions matching the third derivatives of
// the cubics through the first and last four points, evaluation by
// bisection, 0 outside the source range.  Every operation is the one numpy
// performs on complex128 values in pulsesuite_b200.wirespace: complex
// multiply (ar br - ai bi, ar bi + ai br), numpy's complex divide (Smith's
// method with its branch on |br| >= |bi|), real operands taken as (x, 0),
// and no contraction into fused multiply-adds (built with -ffp-contract=off),
// so the results are the same bits as the numpy restatement -- which is
// itself pinned to the reference's outputs.
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "../../include/pulsesuite_b200.h"

namespace {

struct cx {
  double r, i;
};
inline cx cadd(cx a, cx b) { return {a.r + b.r, a.i + b.i}; }
inline cx csub(cx a, cx b) { return {a.r - b.r, a.i - b.i}; }
inline cx cmul(cx a, cx b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
inline cx cneg(cx a) { return {-a.r, -a.i}; }
inline cx real(double x) { return {x, 0.0}; }
// numpy's complex128 division (Smith's method)
inline cx cdiv(cx a, cx b) {
  const double br = fabs(b.r), bi = fabs(b.i);
  if (br >= bi) {
    if (br == 0.0 && bi == 0.0) return {a.r / br, a.i / br};
    const double rat = b.i / b.r;
    const double scl = 1.0 / (b.r + b.i * rat);
    return {(a.r + a.i * rat) * scl, (a.i - a.r * rat) * scl};
  }
  const double rat = b.r / b.i;
  const double scl = 1.0 / (b.i + b.r * rat);
  return {(a.r * rat + a.i) * scl, (a.i * rat - a.r) * scl};
}

int locate(const double* xx, int n, double x) {
  if (x < xx[0]) return 0;
  if (x >= xx[n - 1]) return n - 1;
  int jl = 0, ju = n;
  while (ju - jl > 1) {
    const int jm = (ju + jl) / 2;
    if (x >= xx[jm])
      jl = jm;
    else
      ju = jm;
  }
  return jl;
}

// (b, c, d) of one signal y[n] on x[n]: the numpy restatement line by line
void spline(const double* x, int n, const cx* y, cx* b, cx* c, cx* d) {
  for (int i = 0; i < n; ++i) b[i] = c[i] = d[i] = cx{0.0, 0.0};
  if (n < 3) {
    b[0] = cdiv(csub(y[1], y[0]), real(x[1] - x[0]));
    b[1] = b[0];
    return;
  }
  d[0] = real(x[1] - x[0]);
  c[1] = cdiv(csub(y[1], y[0]), d[0]);
  for (int i = 1; i < n - 1; ++i) {
    d[i] = real(x[i + 1] - x[i]);
    b[i] = cmul(real(2.0), cadd(d[i - 1], d[i]));
    c[i + 1] = cdiv(csub(y[i + 1], y[i]), d[i]);
    c[i] = csub(c[i + 1], c[i]);
  }
  b[0] = cneg(d[0]);
  b[n - 1] = cneg(d[n - 2]);
  c[0] = cx{0.0, 0.0};
  c[n - 1] = cx{0.0, 0.0};
  if (n != 3) {
    c[0] = csub(cdiv(c[2], real(x[3] - x[1])), cdiv(c[1], real(x[2] - x[0])));
    c[n - 1] = csub(cdiv(c[n - 2], real(x[n - 1] - x[n - 3])),
                    cdiv(c[n - 3], real(x[n - 2] - x[n - 4])));
    c[0] = cdiv(cmul(c[0], cmul(d[0], d[0])), real(x[3] - x[0]));
    c[n - 1] = cdiv(cmul(cneg(c[n - 1]), cmul(d[n - 2], d[n - 2])), real(x[n - 1] - x[n - 4]));
  }
  for (int i = 1; i < n; ++i) {
    const cx t = cdiv(d[i - 1], b[i - 1]);
    b[i] = csub(b[i], cmul(t, d[i - 1]));
    c[i] = csub(c[i], cmul(t, c[i - 1]));
  }
  c[n - 1] = cdiv(c[n - 1], b[n - 1]);
  for (int i = n - 2; i >= 0; --i) c[i] = cdiv(csub(c[i], cmul(d[i], c[i + 1])), b[i]);
  b[n - 1] = cadd(cdiv(csub(y[n - 1], y[n - 2]), d[n - 2]),
                  cmul(d[n - 2], cadd(c[n - 2], cmul(real(2.0), c[n - 1]))));
  for (int i = 0; i < n - 1; ++i) {
    b[i] = csub(cdiv(csub(y[i + 1], y[i]), d[i]),
                cmul(d[i], cadd(c[i + 1], cmul(real(2.0), c[i]))));
    d[i] = cdiv(csub(c[i + 1], c[i]), d[i]);
    c[i] = cmul(real(3.0), c[i]);
  }
  c[n - 1] = cmul(real(3.0), c[n - 1]);
  d[n - 1] = d[n - 2];
}

}  // namespace

extern "C" int psb_spline_rows_c128(const double* x0, int n0, const double* z0, int m,
                                    const double* x1, int n1, double* out) {
  if (!x0 || !z0 || !x1 || !out || n0 < 2 || m < 0 || n1 < 0) return PSB_ERR_INVALID;
  double lo = x0[0], hi = x0[0];
  for (int i = 1; i < n0; ++i) {
    lo = x0[i] < lo ? x0[i] : lo;
    hi = x0[i] > hi ? x0[i] : hi;
  }
  // per output point: the interval and its offset, shared by every row
  std::vector<int> jx(n1);
  std::vector<double> dx(n1);
  for (int i = 0; i < n1; ++i) {
    const double u = x1[i];
    jx[i] = (lo <= u && u <= hi) ? locate(x0, n0, u) : -1;
    dx[i] = jx[i] >= 0 ? u - x0[jx[i]] : 0.0;
  }
  // rows are independent: split them over host threads when there are many
  auto rows = [&](int r0, int r1) {
    std::vector<cx> b(n0), c(n0), d(n0);
    for (int r = r0; r < r1; ++r) {
      const cx* y = reinterpret_cast<const cx*>(z0) + (size_t)r * n0;
      cx* o = reinterpret_cast<cx*>(out) + (size_t)r * n1;
      spline(x0, n0, y, b.data(), c.data(), d.data());
      for (int i = 0; i < n1; ++i) {
        const int j = jx[i];
        if (j < 0) {
          o[i] = cx{0.0, 0.0};
          continue;
        }
        const cx h = real(dx[i]);
        o[i] = cadd(y[j], cmul(h, cadd(b[j], cmul(h, cadd(c[j], cmul(h, d[j]))))));
      }
    }
  };
  const long work = (long)m * (n0 + n1);
  int nt = (int)std::min<long>(std::max(1u, std::thread::hardware_concurrency()), 16);
  nt = (int)std::min<long>(nt, std::max<long>(1, work / 4096));
  if (nt <= 1) {
    rows(0, m);
    return PSB_OK;
  }
  std::vector<std::thread> pool;
  const int per = (m + nt - 1) / nt;
  int done = 0;  // rows [0, done) handed to threads
  try {
    for (int t = 0; t < nt; ++t) {
      const int r0 = t * per, r1 = std::min(m, r0 + per);
      if (r0 < r1) pool.emplace_back(rows, r0, r1);
      done = r1;
    }
  } catch (...) {
    // no thread could be started: the remaining rows run here
  }
  if (done < m) rows(done, m);
  for (auto& th : pool) th.join();
  return PSB_OK;
}
