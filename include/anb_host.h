/*
 * anb_host.h - C ABI of the host-side front end in libanb.so: polyMesh I/O and geometry,
 * synthetic channel meshes, the .bc runtime boundary conditions and the VTU writer.
 *
 * These replace the reference's host code that sits in front of and behind the solver:
 *   anb_mesh_read_polymesh      read_openfoam_polymesh      apps/generic_simple_v1/src/main.cu:532-599
 *   anb_mesh_geometry           (geometry part of the same) main.cu:591-597
 *   anb_bc_evaluate             load_runtime_bc_config + build_patch_geometry_table +
 *                               apply_bc_specs_to_legacy_face_arrays
 *                               apps/generic_simple_v1/src/{bc_runtime_config.cu:83-230,
 *                               patch_geometry.cu:84-140, velocity_bc_eval.cu:197-290}
 *   anb_write_vtu               write_vtu_polyhedron_cell_data main.cu:975-983
 *   anb_mesh_make_channel       no counterpart (synthetic benchmark meshes)
 * All functions return 0 on success, non-zero on error with the message in errbuf.
 */
#ifndef ANB_HOST_H
#define ANB_HOST_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct anb_hmesh anb_hmesh;

int anb_mesh_read_polymesh(const char* dir, anb_hmesh** out, char* errbuf, int errlen);
int anb_mesh_make_channel(int nx, int ny, int nz, double lx, double ly, double lz, double jitter,
                          unsigned long long seed, int obstacle, int tets, anb_hmesh** out, char* errbuf,
                          int errlen);
int anb_mesh_write_polymesh(const anb_hmesh* m, const char* dir, char* errbuf, int errlen);
void anb_mesh_free(anb_hmesh* m);

/* n_points, n_faces, n_face_points, n_internal_faces, n_cells, n_patches */
void anb_mesh_sizes(const anb_hmesh* m, int* sizes6);
/* any pointer may be NULL */
void anb_mesh_topology(const anb_hmesh* m, double* points, int* face_offsets, int* face_points, int* owner,
                       int* neighbour, int* patch_start, int* patch_size);
const char* anb_mesh_patch_name(const anb_hmesh* m, int patch);
/* computes the geometry if needed; cc,xf,nf,sf: 3 per entry */
int anb_mesh_geometry(anb_hmesh* m, double* cc, double* vol, double* xf, double* nf, double* sf, double* af,
                      double* max_nonorth, char* errbuf, int errlen);

/* Loads a .bc file and evaluates per-patch types (1 Dirichlet / 0 Neumann) and per-face values
 * (nFaces each).  patch_table (may be NULL): per patch 10 doubles: area, centroid[3],
 * averageNormal[3], planarity, nFaces, sumSf magnitude. */
int anb_bc_evaluate(anb_hmesh* m, const char* bc_path, int* type_u, int* type_v, int* type_w, int* type_p,
                    double* u, double* v, double* w, double* p, double* patch_table, char* errbuf, int errlen);

/* Expands argv with `-case-config` like the reference and writes the resulting argument vector,
 * NUL-separated, into out (returns the count or -1 with the message in errbuf). */
int anb_expand_case_args(int argc, const char* const* argv, char* out, int outlen, char* errbuf, int errlen);

/* ASCII VTU of cell data (U vector + p, umag, cell_volume, divCorr). */
int anb_write_vtu(anb_hmesh* m, const char* filename, const double* u, const double* v, const double* w,
                  const double* p, const double* div_corr, char* errbuf, int errlen);

/* The same VTU with every array as raw little-endian binary in one appended block
 * (<AppendedData encoding="raw">, header_type UInt64): exact values, no text formatting.  No
 * counterpart in the reference, whose writer is ASCII only (main.cu:975-983); the drop-in program
 * selects it with the .case key anbVtuFormat binary. */
int anb_write_vtu_binary(anb_hmesh* m, const char* filename, const double* u, const double* v, const double* w,
                         const double* p, const double* div_corr, char* errbuf, int errlen);

#ifdef __cplusplus
}
#endif
#endif
