/* Host side of the wire <-> volume coupling blocks (dielectric_wire.c's
 * dw_assemble_wire_to_volume and the wire-row loop of
 * dielectric_solve_conductor_coupled) and of the wire MoM fill (matrix.c
 * cmset): argument checks, the Gauss rules, the basis lists, the uploads and
 * downloads around the device kernels of coupling.cu and mom_fill.cu.  C,
 * like the reference. */
#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/nec2c_cuda.h"
#include "../csrc/device_api.h"

#define COUPLING_EPSILON_0 8.8541878128e-12
#define COUPLING_PI 3.141592653589793238462643383279502884

/* Gauss-Legendre nodes and weights on [-1, 1] by Newton's method on the
   Legendre recurrence from the starting guesses cos(pi (i + 3/4) / (n + 1/2)),
   the rule dielectric_wire.c:70-97 builds for its cell averages. */
static int gauss_rule(int order, double *node, double *weight)
{
  int root;
  for(root = 0; root < (order + 1) / 2; ++root) {
    double z = cos(COUPLING_PI * ((double)root + 0.75) / ((double)order + 0.5)), previous, slope = 0.0;
    int iteration = 0;
    do {
      double p0 = 1.0, p1 = z;
      int degree;
      previous = z;
      for(degree = 2; degree <= order; ++degree) {
        const double p2 = (((2.0 * degree) - 1.0) * z * p1 - ((double)degree - 1.0) * p0) / degree;
        p0 = p1;
        p1 = p2;
      }
      slope = order * (z * p1 - p0) / (z * z - 1.0);
      z = previous - p1 / slope;
      ++iteration;
    } while(fabs(z - previous) > 4.0 * DBL_EPSILON && iteration < 32);
    if(iteration == 32) return 0;
    node[root] = -z;
    node[order - 1 - root] = z;
    weight[root] = 2.0 / ((1.0 - z * z) * slope * slope);
    weight[order - 1 - root] = weight[root];
  }
  return 1;
}

static void *upload_new(const void *host, size_t bytes)
{
  void *d = n2d_alloc_async(bytes ? bytes : 16);
  if(d && bytes && !n2d_upload(d, host, bytes)) { n2d_free_async(d); return NULL; }
  return d;
}

static int cells_ok(size_t cells, const double *centers, const double *sizes)
{
  size_t i;
  for(i = 0; i < 3 * cells; ++i)
    if(!isfinite(centers[i]) || !isfinite(sizes[i]) || !(sizes[i] > 0)) return 0;
  return 1;
}

int nec2c_cuda_coupling_wire_to_volume(const nec2c_cuda_wire_model *w, size_t columns,
                                       const nec2c_cuda_complex *sources, size_t cells,
                                       const double *centers, const double *sizes,
                                       const nec2c_cuda_complex *chi, double omega, nec2c_cuda_complex *out)
{
  double node[6], weight[6], *seg = NULL;
  void *seg_d = NULL, *src_d = NULL, *ctr_d = NULL, *sz_d = NULL, *chi_d = NULL, *node_d = NULL, *wt_d = NULL;
  void *out_d = NULL;
  size_t i;
  int ok;
  if(!w || !out || (columns && (!sources || !w->x || !w->y || !w->z || !w->length || !w->radius || !w->cab ||
                                !w->sab || !w->salp)) || (cells && (!centers || !sizes || !chi)) ||
     w->segments == 0 || w->segments > 1000000 || columns > 1000000 || cells > ((size_t)1 << 40) ||
     !(w->wavelength > 0) || !(w->rkh > 0) || !(omega > 0) || (w->pec_ground != 0 && w->pec_ground != 1)) {
    n2c_set_error("wire-to-volume coupling: invalid arguments");
    return 0;
  }
  if(columns == 0 || cells == 0) return 1;
  if(!cells_ok(cells, centers, sizes)) { n2c_set_error("wire-to-volume coupling: invalid cell"); return 0; }
  if(!n2d_device_ok()) return 0;
  if(!gauss_rule(6, node, weight)) { n2c_set_error("wire-to-volume coupling: Gauss rule failed"); return 0; }
  seg = malloc(8 * w->segments * sizeof(double));
  if(!seg) { n2c_set_error("host allocation failed"); return 0; }
  for(i = 0; i < w->segments; ++i) {
    double *g = seg + 8 * i;
    g[0] = w->x[i]; g[1] = w->y[i]; g[2] = w->z[i]; g[3] = w->length[i]; g[4] = w->radius[i];
    g[5] = w->cab[i]; g[6] = w->sab[i]; g[7] = w->salp[i];
  }
  seg_d = upload_new(seg, 8 * w->segments * sizeof(double));
  src_d = upload_new(sources, columns * 3 * w->segments * sizeof(nec2c_cuda_complex));
  ctr_d = upload_new(centers, 3 * cells * sizeof(double));
  sz_d = upload_new(sizes, 3 * cells * sizeof(double));
  chi_d = upload_new(chi, cells * sizeof(nec2c_cuda_complex));
  node_d = upload_new(node, sizeof(node));
  wt_d = upload_new(weight, sizeof(weight));
  out_d = n2d_alloc_async(columns * 3 * cells * sizeof(nec2c_cuda_complex));
  ok = seg_d && src_d && ctr_d && sz_d && chi_d && node_d && wt_d && out_d &&
       n2d_coupling_wire_to_volume(seg_d, (int)w->segments, w->rkh, w->pec_ground, w->wavelength, src_d,
                                   (int)columns, ctr_d, sz_d, chi_d, (long long)cells,
                                   omega * COUPLING_EPSILON_0, node_d, wt_d, out_d) &&
       n2d_download(out, out_d, columns * 3 * cells * sizeof(nec2c_cuda_complex));
  n2d_free_async(seg_d); n2d_free_async(src_d); n2d_free_async(ctr_d); n2d_free_async(sz_d);
  n2d_free_async(chi_d); n2d_free_async(node_d); n2d_free_async(wt_d); n2d_free_async(out_d);
  free(seg);
  return ok;
}

int nec2c_cuda_coupling_volume_to_wire(size_t segments, const double *centers_m, const double *tangents,
                                       size_t cells, const double *cell_centers, const double *cell_sizes,
                                       double k0, double omega, int pec_ground, nec2c_cuda_complex *out)
{
  double node[10], weight[10];
  void *obs_d = NULL, *tan_d = NULL, *ctr_d = NULL, *sz_d = NULL, *node_d = NULL, *wt_d = NULL, *out_d = NULL;
  size_t i;
  int ok;
  if(!out || (segments && (!centers_m || !tangents)) || (cells && (!cell_centers || !cell_sizes)) ||
     segments > 1000000 || cells > ((size_t)1 << 40) || !(k0 >= 0) || !isfinite(k0) || !(omega > 0) ||
     (pec_ground != 0 && pec_ground != 1)) {
    n2c_set_error("volume-to-wire coupling: invalid arguments");
    return 0;
  }
  if(segments == 0 || cells == 0) return 1;
  if(!cells_ok(cells, cell_centers, cell_sizes)) { n2c_set_error("volume-to-wire coupling: invalid cell"); return 0; }
  for(i = 0; i < 3 * segments; ++i)
    if(!isfinite(centers_m[i]) || !isfinite(tangents[i])) {
      n2c_set_error("volume-to-wire coupling: invalid segment");
      return 0;
    }
  if(!n2d_device_ok()) return 0;
  if(!gauss_rule(10, node, weight)) { n2c_set_error("volume-to-wire coupling: Gauss rule failed"); return 0; }
  obs_d = upload_new(centers_m, 3 * segments * sizeof(double));
  tan_d = upload_new(tangents, 3 * segments * sizeof(double));
  ctr_d = upload_new(cell_centers, 3 * cells * sizeof(double));
  sz_d = upload_new(cell_sizes, 3 * cells * sizeof(double));
  node_d = upload_new(node, sizeof(node));
  wt_d = upload_new(weight, sizeof(weight));
  out_d = n2d_alloc_async(segments * 3 * cells * sizeof(nec2c_cuda_complex));
  ok = obs_d && tan_d && ctr_d && sz_d && node_d && wt_d && out_d &&
       n2d_coupling_volume_to_wire(obs_d, tan_d, (int)segments, ctr_d, sz_d, (long long)cells, k0,
                                   omega * COUPLING_EPSILON_0, pec_ground, node_d, wt_d, out_d) &&
       n2d_download(out, out_d, segments * 3 * cells * sizeof(nec2c_cuda_complex));
  n2d_free_async(obs_d); n2d_free_async(tan_d); n2d_free_async(ctr_d); n2d_free_async(sz_d);
  n2d_free_async(node_d); n2d_free_async(wt_d); n2d_free_async(out_d);
  return ok;
}

int nec2c_cuda_mom_fill(const nec2c_cuda_wire_model *w, const size_t *basis_first, const int *basis_column,
                        const nec2c_cuda_complex *basis_coef, const nec2c_cuda_complex *loads,
                        nec2c_cuda_complex *cm, size_t nrow)
{
  size_t n, total, i, j, k;
  double *seg = NULL;
  int *sup_first = NULL, *sup_src = NULL, *fill = NULL;
  nec2c_cuda_complex *sup_coef = NULL;
  void *seg_d = NULL, *first_d = NULL, *src_d = NULL, *coef_d = NULL, *load_d = NULL, *out_d = NULL;
  int ok;
  if(!w || !cm || !basis_first || w->segments == 0 || w->segments > 65536 || nrow < w->segments ||
     !w->x || !w->y || !w->z || !w->length || !w->radius || !w->cab || !w->sab || !w->salp ||
     !(w->rkh > 0) || (w->pec_ground != 0 && w->pec_ground != 1)) {
    n2c_set_error("MoM fill: invalid arguments");
    return 0;
  }
  n = w->segments;
  total = basis_first[n];
  if(basis_first[0] != 0 || total > 64 * n || (total && (!basis_column || !basis_coef))) {
    n2c_set_error("MoM fill: invalid basis lists");
    return 0;
  }
  for(j = 0; j < n; ++j)
    if(basis_first[j + 1] < basis_first[j]) { n2c_set_error("MoM fill: invalid basis lists"); return 0; }
  for(k = 0; k < total; ++k)
    if(basis_column[k] < 0 || (size_t)basis_column[k] >= n || !isfinite(creal(basis_coef[3 * k])) ||
       !isfinite(cimag(basis_coef[3 * k])) || !isfinite(creal(basis_coef[3 * k + 1])) ||
       !isfinite(cimag(basis_coef[3 * k + 1])) || !isfinite(creal(basis_coef[3 * k + 2])) ||
       !isfinite(cimag(basis_coef[3 * k + 2]))) {
      n2c_set_error("MoM fill: invalid basis entry %zu", k);
      return 0;
    }
  for(i = 0; i < n; ++i)
    if(!isfinite(w->x[i]) || !isfinite(w->y[i]) || !isfinite(w->z[i]) || !(w->length[i] > 0) ||
       !(w->radius[i] > 0) || !isfinite(w->cab[i]) || !isfinite(w->sab[i]) || !isfinite(w->salp[i]) ||
       (loads && (!isfinite(creal(loads[i])) || !isfinite(cimag(loads[i]))))) {
      n2c_set_error("MoM fill: invalid segment %zu", i);
      return 0;
    }
  if(!n2d_device_ok()) return 0;
  /* The per-source lists transposed to per-column lists, sources increasing
     (the order cmset's source loop adds them in). */
  seg = malloc(8 * n * sizeof(double));
  sup_first = calloc(n + 1, sizeof(int));
  fill = calloc(n, sizeof(int));
  sup_src = malloc((total ? total : 1) * sizeof(int));
  sup_coef = malloc((total ? total : 1) * 3 * sizeof(nec2c_cuda_complex));
  if(!seg || !sup_first || !fill || !sup_src || !sup_coef) {
    free(seg); free(sup_first); free(fill); free(sup_src); free(sup_coef);
    n2c_set_error("host allocation failed");
    return 0;
  }
  for(k = 0; k < total; ++k) sup_first[basis_column[k] + 1]++;
  for(i = 0; i < n; ++i) sup_first[i + 1] += sup_first[i];
  for(j = 0; j < n; ++j)
    for(k = basis_first[j]; k < basis_first[j + 1]; ++k) {
      const size_t b = (size_t)basis_column[k], at = (size_t)sup_first[b] + (size_t)fill[b]++;
      sup_src[at] = (int)j;
      sup_coef[3 * at] = basis_coef[3 * k];
      sup_coef[3 * at + 1] = basis_coef[3 * k + 1];
      sup_coef[3 * at + 2] = basis_coef[3 * k + 2];
    }
  for(i = 0; i < n; ++i) {
    double *g = seg + 8 * i;
    g[0] = w->x[i]; g[1] = w->y[i]; g[2] = w->z[i]; g[3] = w->length[i]; g[4] = w->radius[i];
    g[5] = w->cab[i]; g[6] = w->sab[i]; g[7] = w->salp[i];
  }
  seg_d = upload_new(seg, 8 * n * sizeof(double));
  first_d = upload_new(sup_first, (n + 1) * sizeof(int));
  src_d = upload_new(sup_src, total * sizeof(int));
  coef_d = upload_new(sup_coef, 3 * total * sizeof(nec2c_cuda_complex));
  load_d = loads ? upload_new(loads, n * sizeof(nec2c_cuda_complex)) : NULL;
  out_d = n2d_alloc_async(n * nrow * sizeof(nec2c_cuda_complex));
  ok = seg_d && first_d && src_d && coef_d && (!loads || load_d) && out_d &&
       n2d_mom_fill(seg_d, (int)n, w->rkh, w->pec_ground, first_d, src_d, coef_d, load_d, out_d,
                    (long long)nrow) &&
       n2d_download(cm, out_d, n * nrow * sizeof(nec2c_cuda_complex));
  n2d_free_async(seg_d); n2d_free_async(first_d); n2d_free_async(src_d); n2d_free_async(coef_d);
  n2d_free_async(load_d); n2d_free_async(out_d);
  free(seg); free(sup_first); free(fill); free(sup_src); free(sup_coef);
  return ok;
}
