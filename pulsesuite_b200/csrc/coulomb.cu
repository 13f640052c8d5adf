// coulomb.cu -- Coulomb tables and static screening (FP64).
//
//   psb_coulomb_vint  Vint double sum      pulsesuite/PSTD3D/coulomb.py:69-104, 548-557
//   psb_coulomb_k0    prefactor*K0(|q|a)   (Bessel method of usefulsubs.py:1669-1820)
//   psb_chi1d         1D susceptibility    coulomb.py:580-630
//   psb_screen_f64    eps(q; n1D_w)         coulomb.py:1172-1193, 1218-1230
#include <math.h>

#include "psb_common.cuh"

namespace psb {

// One block per momentum transfer: the (Ny/2+1)^2 double sum of Vint,
// reduced in a fixed tree.  a1/a2 = (alpha*y)^2 are formed per term.
__global__ void __launch_bounds__(256) vint_kernel(const double* __restrict__ qy, int nq,
                                                  const double* __restrict__ y, int ny,
                                                  double alpha1, double alpha2, double delta0,
                                                  double prefactor, double* __restrict__ out) {
  int iq = blockIdx.x;
  if (iq >= nq) return;
  int n1 = ny / 4, n2 = 3 * ny / 4;
  int m = n2 - n1 + 1;
  double kmin = (alpha1 + alpha2) / 4.0;
  double q = fabs(qy[iq]);
  double dk = q > kmin ? q : kmin;
  double dy = y[1] - y[0];
  double mult = alpha1 * alpha2 / kPi * (dy * dy);
  double d02 = delta0 * delta0;
  double acc = 0.0;
  for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
    int i = n1 + idx / m, j = n1 + idx % m;
    double yi = y[i], yj = y[j];
    double a1 = (alpha1 * yi) * (alpha1 * yi);
    double a2 = (alpha2 * yj) * (alpha2 * yj);
    double d = yi - yj;
    double r = sqrt(__dadd_rn(__dmul_rn(d, d), d02));
    double ef = exp(-a1 - a2);
    acc += __dmul_rn(__dmul_rn(ef, mult), bessel_k0_crude(dk * r));
  }
  __shared__ double red[8];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    out[iq] = prefactor * s;
  }
}

__global__ void k0_table_kernel(const double* __restrict__ q, int nq, double radius,
                                double prefactor, double* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  double qi = q[i];
  out[i] = qi == 0.0 ? 0.0 : prefactor * bessel_k0(fabs(qi) * radius);
}

__global__ void chi1d_kernel(const double* __restrict__ qc, int nq, double alpha, double delta0,
                             double mass, double scale, double* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  double R = sqrt((2.0 / alpha) * (2.0 / alpha) + delta0 * delta0);
  out[i] = mass * bessel_k0(qc[i] * R) / qc[i] * scale;
}

__global__ void __launch_bounds__(256) screen_kernel(const PsbTable* __restrict__ tables,
                                                     int ntab, const double* __restrict__ tabdata,
                                                     const PsbWire* __restrict__ wires,
                                                     const double* __restrict__ y,
                                                     double* __restrict__ eps, int ldeps) {
  int w = blockIdx.x;
  int ti = wires[w].table;
  if (ti < 0 || ti >= ntab) return;  // the wire's eps row is left untouched
  PsbTable tb = tables[ti];
  if (tb.nk < 2 || tb.nk > ldeps) return;
  const double* yw = y + 4 * wires[w].off;
  int nk = tb.nk;
  double s = 0.0;
  for (int k = threadIdx.x; k < nk; k += blockDim.x) s += yw[4 * k + 2] + yw[4 * k + 3];
  __shared__ double red[8];
  __shared__ double n1d_s;
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    double n1d = t / 2.0 / tb.L;
    n1d_s = n1d < tb.dens_max ? n1d : tb.dens_max;
  }
  __syncthreads();
  const double* blk = tabdata + tb.off;
  for (int q = threadIdx.x; q < nk; q += blockDim.x)
    eps[(size_t)w * ldeps + q] = eps1d(blk, nk, q, n1d_s);
}

}  // namespace psb

using namespace psb;

extern "C" int psb_coulomb_vint(const double* d_qy, int nq, const double* d_y, int ny,
                                double alpha1, double alpha2, double delta0, double prefactor,
                                double* d_out, void* stream) {
  if (!d_qy || !d_y || !d_out || nq < 0 || ny < 4)
    return set_error(PSB_ERR_INVALID, "psb_coulomb_vint: bad arguments");
  if (nq == 0) return PSB_OK;
  vint_kernel<<<nq, 256, 0, (cudaStream_t)stream>>>(d_qy, nq, d_y, ny, alpha1, alpha2, delta0,
                                                     prefactor, d_out);
  return check_cuda("psb_coulomb_vint");
}

extern "C" int psb_coulomb_k0(const double* d_q, int nq, double radius, double prefactor,
                              double* d_out, void* stream) {
  if (!d_q || !d_out || nq < 0) return set_error(PSB_ERR_INVALID, "psb_coulomb_k0: bad arguments");
  if (nq == 0) return PSB_OK;
  k0_table_kernel<<<(nq + 127) / 128, 128, 0, (cudaStream_t)stream>>>(d_q, nq, radius, prefactor,
                                                                      d_out);
  return check_cuda("psb_coulomb_k0");
}

extern "C" int psb_chi1d(const double* d_qc, int nq, double alpha, double delta0, double mass,
                         double scale, double* d_out, void* stream) {
  if (!d_qc || !d_out || nq < 0) return set_error(PSB_ERR_INVALID, "psb_chi1d: bad arguments");
  if (nq == 0) return PSB_OK;
  chi1d_kernel<<<(nq + 127) / 128, 128, 0, (cudaStream_t)stream>>>(d_qc, nq, alpha, delta0, mass,
                                                                   scale, d_out);
  return check_cuda("psb_chi1d");
}

extern "C" int psb_screen_f64(const PsbTable* d_tables, int ntab, const double* d_tabdata,
                              const PsbWire* d_wires, int nw, const double* d_y, double* d_eps,
                              int ldeps, void* stream) {
  if (!d_tables || !d_tabdata || !d_wires || !d_y || !d_eps || ntab <= 0 || nw < 0 ||
      ldeps < 1)
    return set_error(PSB_ERR_INVALID, "psb_screen_f64: bad arguments");
  if (nw == 0) return PSB_OK;
  screen_kernel<<<nw, 256, 0, (cudaStream_t)stream>>>(d_tables, ntab, d_tabdata, d_wires, d_y, d_eps,
                                                      ldeps);
  return check_cuda("psb_screen_f64");
}
