"""Writes the build copy of the reference's dielectric_wire.c that hands its
two wire <-> volume coupling blocks to the CUDA backend binding.

The coupling is computed by static code inside dielectric_wire.c, which the
link-time wrapping of the other entry points cannot reach, so the drop-in
program compiles a copy of that file with three insertions (each anchored on
a unique line of the reference file, and the script stops if an anchor is
missing):

1. prototypes of the two binding functions (nec2c_cuda_binding.c);
2. at the top of dw_assemble_wire_to_volume (dielectric_wire.c:422-510): the
   wire -> volume block from the binding when a CUDA backend is selected and
   the model is one the GPU kernels cover (the reference's own code runs
   otherwise, and a GPU failure fails the assembly);
3. before the wire-row loop (dielectric_wire.c:1182-1200): the volume -> wire
   rows from the binding, written through the file's own dw_entry; the loop
   then has no tasks left.

Usage: patch_dielectric_wire.py <reference dielectric_wire.c> <output file>
"""
import sys

PROTOTYPES = """/* CUDA backend binding (nec2c_b200/binding/nec2c_cuda_binding.c): the two
   coupling blocks on the GPU when a CUDA backend is selected. */
int nec2c_binding_wire_to_volume(const dielectric_mesh_result *mesh,size_t nw,size_t np,
    size_t conductor_unknowns,const complex double *sources,
    const complex double *wire_background_basis,const complex double *volume_chi,
    double k0,double omega,complex double **result,int *result_mapped,
    size_t *workers_used,int *fell_back);
complex double *nec2c_binding_volume_to_wire(const dielectric_mesh_result *mesh,size_t nw,
    const double *x,const double *y,const double *z,double k0,double omega);
"""

WIRE_TO_VOLUME = """  {
    int handled=nec2c_binding_wire_to_volume(mesh,nw,np,conductor_unknowns,sources,
        wire_background_basis,volume_chi,k0,omega,result,result_mapped,workers_used,fell_back);
    if(handled) return handled>0;
  }
"""

VOLUME_TO_WIRE = """    {
      complex double *gpu_rows=nec2c_binding_volume_to_wire(mesh,nw,x,y,z,k0,omega);
      if(gpu_rows)
      {
        size_t w_,q_;
        for(w_=0;w_<nw;++w_) for(q_=0;q_<3*nc;++q_)
          *dw_entry(system,accelerated,total,w_*total+conductor_unknowns+q_)=gpu_rows[w_*3*nc+q_];
        free(gpu_rows);
        tasks=0;
      }
    }
"""


def insert(text, anchor, addition, before):
    n = text.count(anchor)
    if n != 1:
        raise SystemExit("patch_dielectric_wire.py: anchor found %d times: %r" % (n, anchor[:60]))
    at = text.index(anchor)
    if not before:
        at += len(anchor)
    return text[:at] + addition + text[at:]


def main():
    src, dst = sys.argv[1], sys.argv[2]
    with open(src) as f:
        text = f.read()
    text = insert(text, "#define DW_EPSILON_0 ", PROTOTYPES, before=True)
    text = insert(text, "    size_t *workers_used,int *fell_back)\n{\n", WIRE_TO_VOLUME, before=False)
    text = insert(text, "#ifdef _OPENMP\n#pragma omp parallel for schedule(dynamic,1) if(tasks >= 8)\n#endif\n"
                        "    for(task=0;task<(ptrdiff_t)tasks;++task)\n    {\n"
                        "      size_t wire=(size_t)task/nc,source_cell=(size_t)task%nc;",
                  VOLUME_TO_WIRE, before=True)
    with open(dst, "w") as f:
        f.write(text)


if __name__ == "__main__":
    main()
