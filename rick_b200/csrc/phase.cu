// W-term phase correction fused with the sum over w-planes.
//
// Replaces phase_g (phase_correction.cu:19-93), which runs one thread per
// (plane, pixel) and adds into the image with FP64 atomics.  Here each thread
// owns one pixel and walks the planes in increasing w, so the image is written
// once, without atomics, and sqrt(1 - l^2 - m^2) is formed once per pixel.
// The phase of plane iw is exp(i * 2*pi*wterm*(sqrt(1-r^2) - 1)) with
// wterm = wmin + iw*dw (phase_correction.cu:51-78; the plane's lower edge, as in
// the reference), in FP64.  l = sin(x*resolution) and m = sin(y*resolution)
// (phase_correction.cu:56-61) come from 1-D tables built on the host with the
// C library's sin, and every rounding up to the phase argument is an explicit
// round-to-nearest operation: sqrt(1-r^2) - 1 loses up to ~14 digits near the
// image centre, so the argument must be the reference's to the last bit.  The
// FFT's 1/(Nx*Ny) scale (fourier_transform.c:24,73-74) is folded into the load.
#include "rick_internal.h"

namespace rick {

namespace {

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

template <typename InT>
__global__ void __launch_bounds__(256)
    k_phase_sum(const typename Vec2<InT>::type *__restrict__ cube, int xaxis, int yaxis, int nw,
                int w_first, int nw_total,
                const double *__restrict__ ltab, const double *__restrict__ mtab, double wmin,
                double dw, double dwnorm, double norm, int phase_on, int accumulate,
                double *__restrict__ img_re, double *__restrict__ img_im) {
  const uint64_t plane = (uint64_t)xaxis * yaxis;
  const uint64_t pix = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (pix >= plane) return;
  const int iv = (int)(pix / xaxis);
  const int iu = (int)(pix % xaxis);
  double acc_re = accumulate ? img_re[pix] : 0.0;
  double acc_im = accumulate ? img_im[pix] : 0.0;
  if (phase_on && nw_total > 1) {
    const double l = ltab[iu], m = mtab[iv];
    const double radius2 = __dadd_rn(__dmul_rn(l, l), __dmul_rn(m, m));
    const double root = __dsqrt_rn(__dsub_rn(1.0, radius2));
    const double rootm1 = __dsub_rn(root, 1.0);
    const double twopi = 2.0 * kPi;  // exact doubling
#pragma unroll 4
    for (int iw = 0; iw < nw; iw++) {
      const double wterm = __dadd_rn(wmin, __dmul_rn((double)(w_first + iw), dw));
      const double arg = __dmul_rn(__dmul_rn(twopi, wterm), rootm1);
      double s, c;
      sincos(arg, &s, &c);
      const auto gv = cube[(uint64_t)iw * plane + pix];
      const double p = __dmul_rn(norm, (double)gv.x), q = __dmul_rn(norm, (double)gv.y);
      acc_re += (p * c - q * s) * dwnorm * root;
      acc_im += (p * s + q * c) * dwnorm * root;
    }
  } else {
    for (int iw = 0; iw < nw; iw++) {
      const auto gv = cube[(uint64_t)iw * plane + pix];
      acc_re += norm * (double)gv.x;
      acc_im += norm * (double)gv.y;
    }
  }
  img_re[pix] = acc_re;
  img_im[pix] = acc_im;
}

}  // namespace

// phase_correction.cu:56-61 on the host: l[iu] = sin(x(iu)*resolution) with
// x(iu) = iu - N/2, shifted by +N when negative.
void phase_tables(int xaxis, int yaxis, int xaxistot, int yaxistot, double resolution,
                  double *l, double *m) {
  for (int iu = 0; iu < xaxis; iu++) {
    double x = (double)(iu - xaxistot / 2);
    if (x < 0.0) x = (double)(iu + xaxistot / 2);
    l[iu] = sin(x * resolution);
  }
  for (int iv = 0; iv < yaxis; iv++) {
    double y = (double)(iv - yaxistot / 2);
    if (y < 0.0) y = (double)(iv + yaxistot / 2);
    m[iv] = sin(y * resolution);
  }
}

int phase_sum(int precision, const void *cube, int xaxis, int yaxis, int nw, int w_first,
              int nw_total, const double *ltab, const double *mtab, double wmin, double wmax,
              double norm, int phase_on, int accumulate, double *img_re, double *img_im,
              cudaStream_t st) {
  // phase_correction.cu:100-102 (the whole cube's plane spacing)
  const double dw = (wmax - wmin) / (double)nw_total;
  const double dwnorm = dw / (wmax - wmin);
  const uint64_t plane = (uint64_t)xaxis * yaxis;
  if (plane == 0) return RICK_OK;
  const unsigned blocks = (unsigned)((plane + 255) / 256);
  if (precision == RICK_PREC_FP64)
    k_phase_sum<double><<<blocks, 256, 0, st>>>((const double2 *)cube, xaxis, yaxis, nw, w_first,
                                                nw_total, ltab,
                                                mtab, wmin, dw, dwnorm, norm, phase_on,
                                                accumulate, img_re, img_im);
  else
    k_phase_sum<float><<<blocks, 256, 0, st>>>((const float2 *)cube, xaxis, yaxis, nw, w_first,
                                               nw_total, ltab, mtab,
                                               wmin, dw, dwnorm, norm, phase_on, accumulate,
                                               img_re, img_im);
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

}  // namespace rick
