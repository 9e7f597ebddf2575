/*
 * rick_oracle.c -- CPU restatement of RICK's imaging hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: only tests/,
 * __graft_entry__.smoke() and the cpu_baseline / reference legs of bench.py
 * load it, and only as the checker or the timed CPU baseline.  The product
 * (rick_b200/csrc, librick_b200.so) never links or calls it.
 *
 * It restates, with 64-bit indices, the reference's CPU path for one rank:
 *   - kernel tables        w-stacking.cu:28-89  (Gaussian, Kaiser-Bessel)
 *   - wstack (CPU branch)  w-stacking.cu:211-270, 438-536
 *   - phase_correction     phase_correction.cu:97-102, 185-250 (PHASE_ON)
 *   - NORMALIZE_UVW        gridding.c:21-83 (one rank)
 *   - one-rank row choice  init.c:335-340 (last 1000 rows dropped),
 *                          gridding.c:139-188 (sector-0 membership incl. the
 *                          v-halo rule), gridding_cpu.c:118 (reverse packing)
 * The FFT between wstack and phase_correction (fourier_transform.c:13-93,
 * FFTW_BACKWARD scaled by 1/(Nx*Ny)) is done by numpy in oracle/oracle.py.
 *
 * Expression order inside each cell update follows the reference so that a
 * single-threaded run is bit-identical to the reference compiled from its own
 * sources (oracle/Makefile builds those into oracle/_ref).  Where the
 * reference has undefined behaviour (32-bit index overflow, grid_w == Nw rows
 * written past the cube, negative footprint bounds wrapping as unsigned) this
 * restatement uses 64-bit indices and skips the row, counting it as dropped.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* allvars.h:47 / w-stacking.h:6 -- the truncated literal; parity needs it */
#define ORACLE_PI 3.14159265359

enum { ORACLE_GAUSS = 0, ORACLE_GAUSS_HI_PRECISION = 1, ORACLE_KAISER_BESSEL = 2 };

/* w-stacking.cu:252-256: oversampling of the 1-D tables and the Gaussian width */
#define ORACLE_INCREASE_PRECISION 5
#define ORACLE_STD22 0.5 /* 1/(2*std*std), std = 1 */

/* Gaussian table, w-stacking.cu:35-51.  n = 5*w_support entries centred on n/2. */
void oracle_make_gauss_table(double *tab, int w_support)
{
  const int n = ORACLE_INCREASE_PRECISION * w_support;
  const int mid = n / 2;
  const double norm = ORACLE_STD22 / ORACLE_PI;
  for (int i = 0; i <= mid; i++) {
    double term = (double)i / (double)ORACLE_INCREASE_PRECISION;
    tab[mid + i] = sqrt(norm) * exp(-(term * term) * ORACLE_STD22);
  }
  for (int i = 0; i < mid; i++) tab[i] = tab[n - 1 - i];
}

/* Unnormalised I0 power series to relative precision `prec`, w-stacking.cu:54-64 */
double oracle_bessel0(double x, double prec)
{
  double d = 0.0, term = 1.0, sum = 1.0;
  do {
    d += 2.0;
    term *= x * x / (d * d);
    sum += term;
  } while (term > sum * prec);
  return sum;
}

/* Kaiser-Bessel table, w-stacking.cu:65-89 with alpha = 8.6, oversampling 1,
 * no sinc (w-stacking.cu:263-266). */
void oracle_make_kb_table(double *tab, int w_support)
{
  const int n = ORACLE_INCREASE_PRECISION * w_support;
  const int mid = n / 2;
  const double alpha = 8.6, oversampling = 1.0;
  const double filter_ratio = 1.0 / oversampling;
  const double norm_factor = oversampling / oracle_bessel0(alpha, 1e-8);
  for (int i = 0; i <= mid; i++) {
    double term = (double)i / mid;
    tab[mid + i] = filter_ratio * oracle_bessel0(alpha * sqrt(1.0 - (term * term)), 1e-8) * norm_factor;
  }
  for (int i = 0; i < mid; i++) tab[i] = tab[n - 1 - i];
}

/* Number of rows that wstack would touch out of bounds and that both this
 * oracle and the product skip (grid_w outside [0,Nw), footprint bounds that
 * would wrap).  Returned through *dropped. */
int oracle_wstack(int kernel, int num_w_planes, uint64_t num_points, uint32_t freq_per_chan,
                  uint32_t polarizations, const double *uu, const double *vv, const double *ww,
                  const float *vis_real, const float *vis_img, const float *weight, double dx,
                  double dw, int w_support, int grid_size_x, int grid_size_y, double *grid,
                  int num_threads, uint64_t *dropped)
{
  const int KernelLen = (w_support - 1) / 2;
  const int increaseprecision = ORACLE_INCREASE_PRECISION;
  const double std22 = ORACLE_STD22;
  const double norm = std22 / ORACLE_PI;
  const int ntab = increaseprecision * w_support;
  double *tab = (double *)malloc((size_t)ntab * sizeof(double));
  if (!tab) return -1;
  if (kernel == ORACLE_GAUSS) oracle_make_gauss_table(tab, w_support);
  else if (kernel == ORACLE_KAISER_BESSEL) oracle_make_kb_table(tab, w_support);

  const int64_t Nx = grid_size_x, Ny = grid_size_y;
  uint64_t ndrop = 0;

#ifdef _OPENMP
  if (num_threads > 0) omp_set_num_threads(num_threads);
#pragma omp parallel for schedule(static) reduction(+ : ndrop)
#endif
  for (int64_t i = 0; i < (int64_t)num_points; i++) {
    const uint64_t visindex = (uint64_t)i * freq_per_chan * polarizations;
    /* w-stacking.cu:464-470: FP64 division then truncation toward zero */
    const double pos_u = uu[i] / dx;
    const double pos_v = vv[i] / dx;
    const double ww_i = ww[i] / dw;
    const int grid_w = (int)ww_i;
    const int grid_u = (int)pos_u;
    const int grid_v = (int)pos_v;
    if (grid_w < 0 || grid_w >= num_w_planes || grid_u < -KernelLen || grid_v < -KernelLen) {
      ndrop++;
      continue;
    }
    /* w-stacking.cu:473-476 expressed as clipping */
    const int64_t jmin = grid_u - KernelLen > 0 ? grid_u - KernelLen : 0;
    const int64_t jmax = grid_u + KernelLen < Nx - 1 ? grid_u + KernelLen : Nx - 1;
    const int64_t kmin = grid_v - KernelLen > 0 ? grid_v - KernelLen : 0;
    const int64_t kmax = grid_v + KernelLen < Ny - 1 ? grid_v + KernelLen : Ny - 1;
    const uint64_t plane_base = (uint64_t)grid_w * (uint64_t)Nx * (uint64_t)Ny;

    for (int64_t k = kmin; k <= kmax; k++) {
      const double v_dist = (double)k + 0.5 - pos_v;
      for (int64_t j = jmin; j <= jmax; j++) {
        const double u_dist = (double)j + 0.5 - pos_u;
        const uint64_t cell = 2 * ((uint64_t)j + (uint64_t)k * (uint64_t)Nx + plane_base);
        double conv_weight;
        if (kernel == ORACLE_GAUSS_HI_PRECISION) {
          /* gauss_kernel_norm, w-stacking.cu:28-33 */
          conv_weight = norm * exp(-((u_dist * u_dist) + (v_dist * v_dist)) * std22);
        } else {
          const int jKer = (int)(increaseprecision * (fabs(u_dist + (double)KernelLen)));
          const int kKer = (int)(increaseprecision * (fabs(v_dist + (double)KernelLen)));
          /* positions >= 0 keep both indices below ntab; the reference reads
           * past its table for u or v in (-dx, 0) -- defined here by clamping */
          conv_weight = tab[jKer < ntab ? jKer : ntab - 1] * tab[kKer < ntab ? kKer : ntab - 1];
        }
        /* w-stacking.cu:508-527: channel-major, polarisation-minor; a sample is
         * skipped when its real part is NaN; weight*vis is a float product. */
        double add_re = 0.0, add_im = 0.0;
        uint64_t ifine = visindex;
        for (uint32_t f = 0; f < freq_per_chan; f++) {
          uint64_t iweight = visindex / freq_per_chan;
          for (uint32_t p = 0; p < polarizations; p++) {
            if (!isnan(vis_real[ifine])) {
              add_re += weight[iweight] * vis_real[ifine] * conv_weight;
              add_im += weight[iweight] * vis_img[ifine] * conv_weight;
            }
            ifine++;
            iweight++;
          }
        }
#ifdef _OPENMP
#pragma omp atomic
#endif
        grid[cell] += add_re;
#ifdef _OPENMP
#pragma omp atomic
#endif
        grid[cell + 1] += add_im;
      }
    }
  }
  free(tab);
  if (dropped) *dropped = ndrop;
  return 0;
}

/* phase_correction.cu:97-102, 185-250 (CPU branch, PHASE_ON) for the planes
 * w_first .. w_first+w_count-1 of a cube of num_w_planes planes: the image
 * accumulates, over those planes, the FFT'd plane times the w-term phase
 * screen times dwnorm*sqrt(1-r^2).  gridss holds only those planes (plane
 * iw at offset (iw - w_first)); dw, dwnorm and wterm are those of the whole
 * cube.  phase_on == 0 or num_w_planes == 1 is a plain sum.  Pixels are
 * processed in any order; for each pixel the planes are summed in increasing
 * iw, which is the reference's order for one thread, and the running sum is
 * read from and written back to the image, so calls over consecutive plane
 * ranges give the bits of one call over all planes. */
int oracle_phase_correction_planes(const double *gridss, double *image_real, double *image_imag,
                                   int xaxis, int yaxis, int num_w_planes, int w_first,
                                   int w_count, int xaxistot, int yaxistot, double resolution,
                                   double wmin, double wmax, int phase_on, int num_threads)
{
  if (w_first < 0 || w_count < 0 || w_first + w_count > num_w_planes) return -1;
  const double dw = (wmax - wmin) / (double)num_w_planes;
  const double dwnorm = dw / (wmax - wmin);
  const int64_t plane = (int64_t)xaxis * (int64_t)yaxis;

#ifdef _OPENMP
  if (num_threads > 0) omp_set_num_threads(num_threads);
#pragma omp parallel for schedule(static)
#endif
  for (int64_t pix = 0; pix < plane; pix++) {
    const int iv = (int)(pix / xaxis);
    const int iu = (int)(pix % xaxis);
    double acc_re = image_real[pix], acc_im = image_imag[pix];
    if (phase_on && num_w_planes > 1) {
      double xcoord = (double)(iu - xaxistot / 2);
      if (xcoord < 0.0) xcoord = (double)(iu + xaxistot / 2);
      xcoord = sin(xcoord * resolution);
      double ycoord = (double)(iv - yaxistot / 2);
      if (ycoord < 0.0) ycoord = (double)(iv + yaxistot / 2);
      ycoord = sin(ycoord * resolution);
      const double radius2 = (xcoord * xcoord + ycoord * ycoord);
      for (int iw = w_first; iw < w_first + w_count; iw++) {
        const double wterm = wmin + iw * dw;
        const double preal = cos(2.0 * ORACLE_PI * wterm * (sqrt(1 - radius2) - 1.0));
        const double pimag = sin(2.0 * ORACLE_PI * wterm * (sqrt(1 - radius2) - 1.0));
        const int64_t index = 2 * (pix + plane * (iw - w_first));
        const double p = gridss[index], q = gridss[index + 1];
        const double r = preal, s = pimag;
        acc_re += (p * r - q * s) * dwnorm * sqrt(1 - radius2);
        acc_im += (p * s + q * r) * dwnorm * sqrt(1 - radius2);
      }
    } else {
      for (int iw = w_first; iw < w_first + w_count; iw++) {
        const int64_t index = 2 * (pix + plane * (iw - w_first));
        acc_re += gridss[index];
        acc_im += gridss[index + 1];
      }
    }
    image_real[pix] = acc_re;
    image_imag[pix] = acc_im;
  }
  return 0;
}

/* The whole cube: phase_correction.cu:97-250 as one call. */
int oracle_phase_correction(const double *gridss, double *image_real, double *image_imag,
                            int xaxis, int yaxis, int num_w_planes, int xaxistot, int yaxistot,
                            double resolution, double wmin, double wmax, int phase_on,
                            int num_threads)
{
  return oracle_phase_correction_planes(gridss, image_real, image_imag, xaxis, yaxis,
                                        num_w_planes, 0, num_w_planes, xaxistot, yaxistot,
                                        resolution, wmin, wmax, phase_on, num_threads);
}

/* Rows that one rank grids, in the order it packs them.
 *  - init.c:337-339: the last 1000 rows of the file are never read;
 *  - gridding.c:149-188 with nsectors = 1, yaxis = grid_size_y: a row belongs to
 *    sector 0 when (int)v == 0, or as a halo row of its neighbour sector when
 *    its distance to the slab edge is in [0, w_supporth);
 *  - gridding_cpu.c:118: sector rows are packed in reverse order.
 * rows_out must hold nmeasures_file entries.  Returns the count (or 0 when the
 * file holds no more than 1000 rows). */
uint64_t oracle_sector0_rows(const double *vv, uint64_t nmeasures_file, int grid_size_x,
                             int grid_size_y, int w_support, uint64_t *rows_out)
{
  if (nmeasures_file <= 1000) return 0;
  const uint64_t nm = nmeasures_file - 1000;
  const int nsectors = 1;
  const int yaxis = grid_size_y / nsectors;
  const double dx = 1.0 / (double)grid_size_x;
  const double w_supporth = (double)((w_support - 1) / 2) * dx;
  uint64_t count = 0;
  for (uint64_t iphi = 0; iphi < nm; iphi++) {
    const double vvh = vv[iphi];
    const int binphi = (int)(vvh * nsectors);
    const double updist = (double)((binphi + 1) * yaxis) * dx - vvh;
    const double downdist = vvh - (double)(binphi * yaxis) * dx;
    int in0 = (binphi == 0);
    if (binphi + 1 == 0 && updist < w_supporth && updist >= 0.0) in0 = 1;
    if (binphi - 1 == 0 && downdist < w_supporth && binphi > 0 && downdist >= 0.0) in0 = 1;
    if (in0) rows_out[count++] = iphi;
  }
  /* reverse: packing walks the sector list from its end */
  for (uint64_t a = 0, b = count ? count - 1 : 0; a < b; a++, b--) {
    uint64_t t = rows_out[a];
    rows_out[a] = rows_out[b];
    rows_out[b] = t;
  }
  return count;
}

/* Gather the chosen rows into contiguous arrays (gridding_cpu.c:121-138). */
void oracle_pack_rows(const uint64_t *rows, uint64_t nrows, uint32_t nchan, uint32_t npol,
                      const double *uu, const double *vv, const double *ww, const float *weights,
                      const float *vis_re, const float *vis_im, double *uus, double *vvs,
                      double *wws, float *weightss, float *visreals, float *visimgs)
{
  const uint64_t nv = (uint64_t)nchan * npol;
  for (uint64_t r = 0; r < nrows; r++) {
    const uint64_t i = rows[r];
    uus[r] = uu[i];
    vvs[r] = vv[i]; /* sector 0: v - 0*shift */
    wws[r] = ww[i];
    memcpy(weightss + r * npol, weights + i * npol, npol * sizeof(float));
    memcpy(visreals + r * nv, vis_re + i * nv, nv * sizeof(float));
    memcpy(visimgs + r * nv, vis_im + i * nv, nv * sizeof(float));
  }
}

/* NORMALIZE_UVW of gridding.c:21-83 for one rank, in place.  The extrema start
 * at 1e20 (minima) and 0 (maxima) as in the reference, so a maximum is never
 * below 0; u and v map to (x + maxg) / (2 maxg) with maxg = 1.001 * the largest
 * |extremum| of u and v, w to (w - wmin) / (wmax - wmin).  extrema[0..6] =
 * min u, min v, min w, max u, max v, max w, maxg.  (Rows whose coordinates are
 * NaN make the reference's result depend on the row order; they are not
 * supported here.) */
void oracle_normalize_uvw(uint64_t n, double *uu, double *vv, double *ww, double *extrema)
{
  double mnu = 1e20, mnv = 1e20, mnw = 1e20, mxu = 0.0, mxv = 0.0, mxw = 0.0;
  for (uint64_t i = 0; i < n; i++) {
    mnu = uu[i] < mnu ? uu[i] : mnu;
    mnv = vv[i] < mnv ? vv[i] : mnv;
    mnw = ww[i] < mnw ? ww[i] : mnw;
    mxu = uu[i] > mxu ? uu[i] : mxu;
    mxv = vv[i] > mxv ? vv[i] : mxv;
    mxw = ww[i] > mxw ? ww[i] : mxw;
  }
  const double offset = 0.001;
  const double ming = fmax(fabs(mnu), fabs(mnv));
  double maxg = fmax(fabs(mxu), fabs(mxv));
  maxg = maxg > ming ? maxg : ming;
  maxg = maxg + offset * maxg;
  for (uint64_t i = 0; i < n; i++) {
    uu[i] = (uu[i] + maxg) / (2.0 * maxg);
    vv[i] = (vv[i] + maxg) / (2.0 * maxg);
    ww[i] = (ww[i] - mnw) / (mxw - mnw);
  }
  if (extrema) {
    extrema[0] = mnu; extrema[1] = mnv; extrema[2] = mnw;
    extrema[3] = mxu; extrema[4] = mxv; extrema[5] = mxw;
    extrema[6] = maxg;
  }
}
