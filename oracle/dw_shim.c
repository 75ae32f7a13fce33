/* Test infrastructure only: access to the reference's own wire <-> volume
 * coupling kernels, which are static functions of dielectric_wire.c.  This
 * file includes that source file (so the statics are visible here) and is
 * linked into oracle/_ref/libdw_shim.so with the other reference objects,
 * dielectric_wire.o left out.  The GPU coupling tests compare the CUDA blocks
 * with these on the same inputs; the product never loads this library.
 *
 * shim_point_cuboid_n       dw_point_cuboid_n (dielectric_wire.c:101-221)
 * shim_wire_to_volume       dw_assemble_wire_to_volume (dielectric_wire.c:422-510),
 *                           serial, with NEC's globals set from the arguments
 */
#include "dielectric_wire.c"

int shim_point_cuboid_n(const double *observation, const double *center, const double *size, double k0,
                        int ksymp, int iperf, double *out18)
{
  dielectric_cell cell;
  complex double r[3][3];
  int p, q, ks = gnd.ksymp, ip = gnd.iperf;
  memset(&cell, 0, sizeof(cell));
  for(p = 0; p < 3; ++p) { cell.center[p] = center[p]; cell.size[p] = size[p]; }
  gnd.ksymp = ksymp;
  gnd.iperf = iperf;
  p = dw_point_cuboid_n(observation, &cell, k0, r);
  gnd.ksymp = ks;
  gnd.iperf = ip;
  if(!p) return 0;
  for(p = 0; p < 3; ++p)
    for(q = 0; q < 3; ++q) { out18[2 * (3 * p + q)] = creal(r[p][q]); out18[2 * (3 * p + q) + 1] = cimag(r[p][q]); }
  return 1;
}

/* seg8: per segment x y z length radius cab sab salp (wavelengths). */
int shim_wire_to_volume(int n, const double *seg8, double wlam, double rkh, int ksymp, int iperf,
                        size_t columns, const complex double *sources, size_t cells, const double *centers,
                        const double *sizes, const complex double *chi, double k0, double omega,
                        complex double *out)
{
  dielectric_mesh_result mesh;
  complex double *result = NULL;
  int mapped = 0, fell_back = 0, ok, i, d;
  size_t workers = 0, c;
  double *arrays = calloc((size_t)14 * n, sizeof(double));
  int *icon = calloc((size_t)2 * n, sizeof(int));
  memset(&mesh, 0, sizeof(mesh));
  mesh.cells = calloc(cells, sizeof(dielectric_cell));
  if(!arrays || !icon || !mesh.cells) { free(arrays); free(icon); free(mesh.cells); return 0; }
  mesh.cell_count = cells;
  for(c = 0; c < cells; ++c)
    for(d = 0; d < 3; ++d) { mesh.cells[c].center[d] = centers[3 * c + d]; mesh.cells[c].size[d] = sizes[3 * c + d]; }
  data.n = n; data.m = 0; data.np = n; data.mp = 0;
  data.x = arrays; data.y = arrays + n; data.z = arrays + 2 * n; data.si = arrays + 3 * n;
  data.bi = arrays + 4 * n; data.cab = arrays + 5 * n; data.sab = arrays + 6 * n; data.salp = arrays + 7 * n;
  crnt.air = arrays + 8 * n; crnt.aii = arrays + 9 * n; crnt.bir = arrays + 10 * n; crnt.bii = arrays + 11 * n;
  crnt.cir = arrays + 12 * n; crnt.cii = arrays + 13 * n;
  data.icon1 = icon; data.icon2 = icon + n;
  for(i = 0; i < n; ++i) {
    data.x[i] = seg8[8 * i]; data.y[i] = seg8[8 * i + 1]; data.z[i] = seg8[8 * i + 2];
    data.si[i] = seg8[8 * i + 3]; data.bi[i] = seg8[8 * i + 4];
    data.cab[i] = seg8[8 * i + 5]; data.sab[i] = seg8[8 * i + 6]; data.salp[i] = seg8[8 * i + 7];
  }
  data.wlam = wlam;
  dataj.rkh = rkh;
  dataj.iexk = 0;
  gnd.ksymp = ksymp;
  gnd.iperf = iperf;
  gnd.frati = 1.0;
  dw_coupling_processes = 1;
  ok = dw_assemble_wire_to_volume(&mesh, (size_t)n, 0, columns, sources, NULL, chi, k0, omega, &result, &mapped,
                                  &workers, &fell_back);
  if(ok) memcpy(out, result, columns * 3 * cells * sizeof(*out));
  if(result) dw_free_coupling(result, columns * 3 * cells, mapped);
  data.x = data.y = data.z = data.si = data.bi = data.cab = data.sab = data.salp = NULL;
  crnt.air = crnt.aii = crnt.bir = crnt.bii = crnt.cir = crnt.cii = NULL;
  data.icon1 = data.icon2 = NULL;
  data.n = 0;
  gnd.ksymp = 1;
  free(arrays); free(icon); free(mesh.cells);
  return ok;
}
