/*
 * rick_imager -- host driver for one GPU, with the flow of the reference's
 * main() (main.c:32-166) for a single rank:
 *
 *   read_parameter_file  (init.c:129-291)   paramfile.txt key/value pairs
 *   for each dataset:
 *     readMetaData        (init.c:300-333)   meta.txt
 *     metaData_calculation(init.c:335-370)   the last 1000 rows are not read
 *     readData            (init.c:413-503)   binMS files
 *     gridding + fftw_data + write_fftw_data -> one rick_plan_image_host call
 *                                             (sector-0 rows, gridding.c:149-188)
 *     WRITE_IMAGE          (fourier_transform.c:281-292) <i>fft_real.bin, <i>fft_img.bin
 *   write_result         (result.c:6-53)   stage times, timings.dat
 *
 * The gridding kernel, precision form, PHASE_ON and NORMALIZE_UVW are
 * compile-time macros in the reference; here they are optional paramfile keys
 * (kernel, precision, phase_on, normalize_uvw) or the RICK_KERNEL /
 * RICK_PRECISION / RICK_PHASE_ON / RICK_NORMALIZE_UVW environment
 * variables, defaulting to the reference Makefile's KAISERBESSEL, FP64, on.
 * Errors print like shutdown_wstacking (main.c:6-28) and exit with the code.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "rick_b200.h"

#define NAME_LEN 1000
#define MAX_DATASETS 100

typedef struct {
  int num_threads, ndatasets, grid_size_x, grid_size_y, num_w_planes, w_support;
  int kernel, precision, phase_on, normalize_uvw, fits;
  char datapath[MAX_DATASETS][NAME_LEN];
  char ufile[NAME_LEN], vfile[NAME_LEN], wfile[NAME_LEN], weightsfile[NAME_LEN];
  char visrealfile[NAME_LEN], visimgfile[NAME_LEN], metafile[NAME_LEN];
  char fftfile2[NAME_LEN], fftfile3[NAME_LEN], timingfile[NAME_LEN];
} params_t;

typedef struct {
  uint64_t Nmeasures, Nvis;
  uint32_t freq_per_chan, polarisations, Ntimes, baselines;
  double dt, thours, uvmin, uvmax, wmin, wmax;
} meta_t;

static double wall(void) {
  struct timespec t;
  clock_gettime(CLOCK_REALTIME, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static void shutdown_rick(int code, const char *msg, int line) {
  if (code > 0)
    printf("an error occurred at line %d of file %s\nerror message is: %s\nerror code is: %d\n",
           line, __FILE__, msg, code);
  exit(code);
}

static int kernel_code(const char *s) {
  if (!strcmp(s, "gauss") || !strcmp(s, "GAUSS")) return RICK_KERNEL_GAUSS;
  if (!strcmp(s, "gauss_hi") || !strcmp(s, "GAUSS_HI_PRECISION")) return RICK_KERNEL_GAUSS_HI_PRECISION;
  if (!strcmp(s, "kaiser_bessel") || !strcmp(s, "KAISERBESSEL")) return RICK_KERNEL_KAISER_BESSEL;
  return -1;
}

/* The FITSIO output of fourier_transform.c:227-279 (parallel_real.fits,
 * parallel_img.fits: a primary array of DOUBLE_IMG, NAXIS1 = Nx, NAXIS2 = Ny,
 * x fastest -- the layout of the .bin images) written directly: 80-character
 * header cards in a 2880-byte block, then big-endian IEEE doubles padded to a
 * 2880-byte boundary.  No cfitsio is needed. */
static int write_fits(const char *name, const double *img, int nx, int ny) {
  FILE *f = fopen(name, "wb");
  if (!f) return -1;
  char hdr[2880];
  memset(hdr, ' ', sizeof(hdr));
  const char *cards[6];
  char c[6][81];
  snprintf(c[0], 81, "%-8s= %20s", "SIMPLE", "T");
  snprintf(c[1], 81, "%-8s= %20d", "BITPIX", -64);
  snprintf(c[2], 81, "%-8s= %20d", "NAXIS", 2);
  snprintf(c[3], 81, "%-8s= %20d", "NAXIS1", nx);
  snprintf(c[4], 81, "%-8s= %20d", "NAXIS2", ny);
  snprintf(c[5], 81, "%-8s= %20s", "EXTEND", "T");
  for (int i = 0; i < 6; i++) {
    cards[i] = c[i];
    memcpy(hdr + 80 * i, cards[i], strlen(cards[i]));
  }
  memcpy(hdr + 80 * 6, "END", 3);
  int ok = fwrite(hdr, 1, sizeof(hdr), f) == sizeof(hdr);
  const uint64_t n = (uint64_t)nx * ny;
  unsigned char buf[8 * 512];
  for (uint64_t i = 0; i < n && ok;) {
    const uint64_t m = (n - i) < 512 ? (n - i) : 512;
    for (uint64_t k = 0; k < m; k++) {
      uint64_t b;
      memcpy(&b, img + i + k, 8);
      for (int byte = 0; byte < 8; byte++) buf[8 * k + byte] = (unsigned char)(b >> (56 - 8 * byte));
    }
    ok = fwrite(buf, 8, m, f) == m;
    i += m;
  }
  const uint64_t used = (8 * n) % 2880;
  if (ok && used) {
    memset(hdr, 0, sizeof(hdr));
    ok = fwrite(hdr, 1, 2880 - used, f) == 2880 - used;
  }
  return (fclose(f) == 0 && ok) ? 0 : -1;
}

static int read_params(const char *fname, params_t *p) {
  memset(p, 0, sizeof(*p));
  p->kernel = RICK_KERNEL_KAISER_BESSEL;
  p->precision = RICK_PREC_FP64;
  p->phase_on = 1;
  strcpy(p->fftfile2, "fft_real.bin");
  strcpy(p->fftfile3, "fft_img.bin");
  strcpy(p->timingfile, "timings.dat");
  FILE *f = fopen(fname, "r");
  if (!f) return RICK_ERR_IN_PARAMFILE;
  char k[NAME_LEN], v[NAME_LEN];
  while (fscanf(f, "%999s %999s", k, v) == 2) {
    if (!strcmp(k, "num_threads")) p->num_threads = atoi(v);
    else if (!strcmp(k, "ndatasets")) p->ndatasets = atoi(v);
    else if (!strcmp(k, "w_support")) p->w_support = atoi(v);
    else if (!strcmp(k, "grid_size_x")) p->grid_size_x = atoi(v);
    else if (!strcmp(k, "grid_size_y")) p->grid_size_y = atoi(v);
    else if (!strcmp(k, "num_w_planes")) p->num_w_planes = atoi(v);
    else if (!strcmp(k, "ufile")) strcpy(p->ufile, v);
    else if (!strcmp(k, "vfile")) strcpy(p->vfile, v);
    else if (!strcmp(k, "wfile")) strcpy(p->wfile, v);
    else if (!strcmp(k, "weightsfile")) strcpy(p->weightsfile, v);
    else if (!strcmp(k, "visrealfile")) strcpy(p->visrealfile, v);
    else if (!strcmp(k, "visimgfile")) strcpy(p->visimgfile, v);
    else if (!strcmp(k, "metafile")) strcpy(p->metafile, v);
    else if (!strcmp(k, "fftfile2")) strcpy(p->fftfile2, v);
    else if (!strcmp(k, "fftfile3")) strcpy(p->fftfile3, v);
    else if (!strcmp(k, "timingfile")) strcpy(p->timingfile, v);
    else if (!strcmp(k, "kernel")) p->kernel = kernel_code(v);
    else if (!strcmp(k, "precision")) p->precision = !strcmp(v, "mixed") ? RICK_PREC_MIXED : RICK_PREC_FP64;
    else if (!strcmp(k, "phase_on")) p->phase_on = atoi(v) != 0;
    else if (!strcmp(k, "normalize_uvw")) p->normalize_uvw = atoi(v) != 0;
    else if (!strcmp(k, "fits")) p->fits = atoi(v) != 0;
    else if (!strncmp(k, "Datapath", 8)) {
      const int i = atoi(k + 8);
      if (i >= 1 && i <= MAX_DATASETS) strcpy(p->datapath[i - 1], v);
    }
  }
  fclose(f);
  const char *e;
  if ((e = getenv("RICK_KERNEL"))) p->kernel = kernel_code(e);
  if ((e = getenv("RICK_PRECISION"))) p->precision = !strcmp(e, "mixed") ? RICK_PREC_MIXED : RICK_PREC_FP64;
  if ((e = getenv("RICK_PHASE_ON"))) p->phase_on = !(strcmp(e, "0") == 0 || strcmp(e, "off") == 0);
  if ((e = getenv("RICK_NORMALIZE_UVW"))) p->normalize_uvw = !(strcmp(e, "0") == 0 || strcmp(e, "off") == 0);
  if (p->ndatasets < 1 || p->ndatasets > MAX_DATASETS || p->grid_size_x <= 0 ||
      p->grid_size_y <= 0 || p->num_w_planes <= 0 || p->w_support <= 0 || p->kernel < 0)
    return RICK_ERR_IN_PARAMFILE;
  return RICK_OK;
}

static int path_join(char *out, const char *dir, const char *file) {
  const int n = snprintf(out, NAME_LEN, "%s%s", dir, file);  /* init.c:294-297 */
  return (n > 0 && n < NAME_LEN) ? 0 : -1;
}

static int read_meta(const char *dir, const char *metafile, meta_t *m) {
  char fn[NAME_LEN];
  if (path_join(fn, dir, metafile)) return RICK_ERR_IO;
  FILE *f = fopen(fn, "r");
  if (!f) return RICK_ERR_IO;
  unsigned long long nm = 0, nv = 0;
  int ret = fscanf(f, "%llu %llu %u %u %u %lf %lf %u %lf %lf %lf %lf", &nm, &nv, &m->freq_per_chan,
                   &m->polarisations, &m->Ntimes, &m->dt, &m->thours, &m->baselines, &m->uvmin,
                   &m->uvmax, &m->wmin, &m->wmax);
  fclose(f);
  if (ret != 12) return RICK_ERR_IO;
  m->Nmeasures = nm;
  m->Nvis = nv;
  return RICK_OK;
}

static int read_file(const char *dir, const char *name, void *dst, size_t bytes) {
  char fn[NAME_LEN];
  if (path_join(fn, dir, name)) return RICK_ERR_IO;
  FILE *f = fopen(fn, "rb");
  if (!f) return RICK_ERR_IO;
  const size_t got = fread(dst, 1, bytes, f);
  fclose(f);
  return got == bytes ? RICK_OK : RICK_ERR_IO;
}

int main(int argc, char **argv) {
  if (argc < 2) {
    fprintf(stderr, "please, specify a parameter file as first argument at command line\n");
    return 1;
  }
  const double t_total = wall();
  params_t P;
  if (read_params(argv[1], &P) != RICK_OK)
    shutdown_rick(RICK_ERR_IN_PARAMFILE, "I/O error while reading paramfile", __LINE__);
  printf("RICK imaging hot path on B200 (rick_imager)\n");
  double t_setup = 0, t_kernel = 0, t_write = 0;
  for (int ids = 0; ids < P.ndatasets; ids++) {
    printf("\nDataset %d\n", ids);
    double t0 = wall();
    meta_t M;
    if (read_meta(P.datapath[ids], P.metafile[0] ? P.metafile : "meta.txt", &M) != RICK_OK)
      shutdown_rick(RICK_ERR_IO, "error opening meta file", __LINE__);
    const uint64_t nsub = 1000;
    const uint64_t nm = M.Nmeasures > nsub ? M.Nmeasures - nsub : 0;
    printf("Subtracting last %llu measurements\n", (unsigned long long)nsub);
    const uint64_t npol = M.polarisations, nv = (uint64_t)M.freq_per_chan * npol;
    printf("N. measurements %llu\nChannels %u\nCorrelations %u\nN. visibilities %llu\n",
           (unsigned long long)nm, M.freq_per_chan, M.polarisations,
           (unsigned long long)(nm * nv));
    double *uu = malloc(nm * 8 + 8), *vv = malloc(nm * 8 + 8), *ww = malloc(nm * 8 + 8);
    float *wt = malloc(nm * npol * 4 + 4);
    if (!uu || !vv || !ww || !wt)
      shutdown_rick(RICK_ERR_NOT_ENOUGH_MEM, "Not enough memory for the dataset", __LINE__);
    const char *dir = P.datapath[ids];
    if (read_file(dir, P.ufile, uu, nm * 8) || read_file(dir, P.vfile, vv, nm * 8) ||
        read_file(dir, P.wfile, ww, nm * 8) || read_file(dir, P.weightsfile, wt, nm * npol * 4))
      shutdown_rick(RICK_ERR_IO, "error reading the binMS files", __LINE__);
    t_setup += wall() - t0;

    t0 = wall();
    rick_plan_desc d;
    memset(&d, 0, sizeof(d));
    d.grid_size_x = P.grid_size_x;
    d.grid_size_y = P.grid_size_y;
    d.num_w_planes = P.num_w_planes;
    d.w_support = P.w_support;
    d.kernel = P.kernel;
    d.precision = P.precision;
    d.phase_on = P.phase_on;
    d.normalize_uvw = P.normalize_uvw;
    d.device = 0;
    d.max_rows = nm ? nm : 1;
    d.freq_per_chan = M.freq_per_chan;
    d.polarizations = M.polarisations;
    rick_plan *plan = NULL;
    int st = rick_plan_create(&plan, &d);
    if (st != RICK_OK) shutdown_rick(st, rick_last_error_message(), __LINE__);
    const double resolution = 1.0 / fmax(fabs(M.uvmin), fabs(M.uvmax));  /* gridding_cpu.c:78 */
    printf("RESOLUTION = %f rad, %f arcsec\n", resolution, (3600.0 * 180.0) * resolution / 3.14159265359);
    const uint64_t plane = (uint64_t)P.grid_size_x * P.grid_size_y;
    double *img_re = calloc(plane, 8), *img_im = calloc(plane, 8);
    if (!img_re || !img_im) shutdown_rick(RICK_ERR_NOT_ENOUGH_MEM, "image allocation", __LINE__);
    /* the samples stream from disk in slices of rows into two pinned buffer pairs:
     * a slice is read while the previous one copies and bins */
    st = rick_plan_ingest_begin(plan, nm, uu, vv, ww, wt, RICK_ROWS_SECTOR0);
    if (st != RICK_OK) shutdown_rick(st, rick_last_error_message(), __LINE__);
    const uint64_t slice = nv ? (64ull << 20) / (nv * 4) + 1 : 1;
    void *buf[2][2] = {{NULL, NULL}, {NULL, NULL}};
    for (int b = 0; b < 2; b++)
      for (int c = 0; c < 2; c++)
        if (rick_host_alloc(&buf[b][c], slice * nv * 4 + 16) != RICK_OK)
          shutdown_rick(RICK_ERR_NOT_ENOUGH_MEM, "pinned sample buffers", __LINE__);
    char fre_in[NAME_LEN], fim_in[NAME_LEN];
    if (path_join(fre_in, dir, P.visrealfile) || path_join(fim_in, dir, P.visimgfile))
      shutdown_rick(RICK_ERR_IO, "binMS path too long", __LINE__);
    FILE *fr_in = fopen(fre_in, "rb"), *fi_in = fopen(fim_in, "rb");
    if (!fr_in || !fi_in) shutdown_rick(RICK_ERR_IO, "error opening the visibility files", __LINE__);
    for (uint64_t r0 = 0, k = 0; r0 < nm; r0 += slice, k++) {
      const uint64_t n = (nm - r0) < slice ? (nm - r0) : slice;
      float *a = buf[k & 1][0], *b = buf[k & 1][1];
      if (fread(a, 4, n * nv, fr_in) != n * nv || fread(b, 4, n * nv, fi_in) != n * nv)
        shutdown_rick(RICK_ERR_IO, "error reading the binMS files", __LINE__);
      st = rick_plan_ingest_samples(plan, r0, n, a, b);
      if (st != RICK_OK) shutdown_rick(st, rick_last_error_message(), __LINE__);
    }
    fclose(fr_in);
    fclose(fi_in);
    st = rick_plan_ingest_end(plan, resolution, M.wmin, M.wmax, img_re, img_im);
    if (st != RICK_OK) shutdown_rick(st, rick_last_error_message(), __LINE__);
    for (int b = 0; b < 2; b++)
      for (int c = 0; c < 2; c++) rick_host_free(buf[b][c]);
    rick_plan_stats stats;
    rick_plan_get_stats(plan, &stats);
    printf("rows gridded %llu, dropped %llu, records %llu\n",
           (unsigned long long)stats.rows_gridded, (unsigned long long)stats.rows_dropped,
           (unsigned long long)stats.records);
    rick_plan_destroy(plan);
    t_kernel += wall() - t0;

    t0 = wall();
    char fre[NAME_LEN], fim[NAME_LEN];
    snprintf(fre, sizeof(fre), "%d%s", ids, P.fftfile2);  /* op_filename, init.c:103-109 */
    snprintf(fim, sizeof(fim), "%d%s", ids, P.fftfile3);
    FILE *fr = fopen(fre, "wb"), *fi = fopen(fim, "wb");
    if (!fr || !fi) shutdown_rick(RICK_ERR_IO, "cannot write the image files", __LINE__);
    fwrite(img_re, 8, plane, fr);
    fwrite(img_im, 8, plane, fi);
    fclose(fr);
    fclose(fi);
    if (P.fits) {  /* fourier_transform.c:227-279, main.c:107-108 */
      /* dataset 0 writes the reference's names; later datasets prefix their index */
      char fre2[64], fim2[64];
      if (ids) {
        snprintf(fre2, sizeof(fre2), "%dparallel_real.fits", ids);
        snprintf(fim2, sizeof(fim2), "%dparallel_img.fits", ids);
      } else {
        snprintf(fre2, sizeof(fre2), "parallel_real.fits");
        snprintf(fim2, sizeof(fim2), "parallel_img.fits");
      }
      if (write_fits(fre2, img_re, P.grid_size_x, P.grid_size_y) ||
          write_fits(fim2, img_im, P.grid_size_x, P.grid_size_y))
        shutdown_rick(RICK_ERR_IO, "cannot write the FITS images", __LINE__);
    }
    t_write += wall() - t0;
    free(uu); free(vv); free(ww); free(wt); free(img_re); free(img_im);
    printf("*************************************************************\n");
  }
  const double total = wall() - t_total;
  printf("%40s time: %g sec\n", "Setup", t_setup);
  printf("%40s time : %g sec\n", "Imaging (sample read+grid+fft+phase)", t_kernel);
  printf("%40s time : %g sec\n", "Image writing", t_write);
  printf("%40s time : %g sec\n", "TOT", total);
  FILE *tf = fopen(P.timingfile, "w");
  if (tf) {
    fprintf(tf, "%g %g %g %g\n", t_setup, t_kernel, t_write, total);
    fclose(tf);
  }
  return 0;
}
