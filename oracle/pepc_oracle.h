/*
 * pepc_oracle.h -- CPU FP64 restatement of PEPC's tree-code force evaluation.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * library libpepcg: only the tests, the smoke check and the CPU-baseline leg of
 * the benchmark may load it.  The product path never calls it.
 *
 * Every function restates a piece of the reference (Fortran, ALaDyn/pepc) and
 * cites the file:line it follows.  Arithmetic is IEEE FP64 in the reference's
 * operation order; the library is compiled with -ffp-contract=off so that no
 * multiply-add is fused behind the reader's back.
 */
#ifndef PEPC_ORACLE_H
#define PEPC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Parameters: the union of the /libpepc/ and /calc_force_coulomb/ namelists that
 * matter for the Coulomb tree code (module_libpepc_main.f90:44,
 * coulomb/module_interaction_specific.f90:35-43), plus the walk variant. */
typedef struct orc_params {
  double theta2;            /* square of the BH opening angle (default 0.36) */
  double eps2;              /* Plummer softening squared (default 0) */
  int32_t curve;            /* 0 = Hilbert (reference), 1 = Morton (extra) */
  int32_t walk;             /* 0 = pthreads (per-target LIFO), 1 = simple (tile), 2 = buckets
                               of tile_size (<= 64) consecutive targets, simple rule */
  int32_t tile_size;        /* simple walk tile size (reference: 16) */
  int32_t force_cubic_domain;
  int32_t periodicity[3];
  int32_t mirror_box_layers;
  int32_t include_far_field_if_periodic;
  int32_t fmm_extrinsic_correction; /* 0 none, 1 Redlack, 2 fictitious charges */
  double t_lattice_1[3], t_lattice_2[3], t_lattice_3[3];
  double lattice_origin[3];
  int32_t num_threads;      /* host threads for the walk (1 = serial) */
  int32_t mac_select;       /* 0 Barnes-Hut, 1 Bmax, other: no acceptance (N^2) */
  int32_t force_law;        /* 3 3D Coulomb, 2 2D Coulomb, 4 Lennard-Jones, 5 Kelbg */
  double kelbg_invsqrttemp; /* Kelbg: 1/sqrt(temperature) [0] */
  double spatial_interaction_cutoff[3]; /* module_mirror_boxes.f90:52 [huge] */
} orc_params;

void orc_params_default(orc_params* p);

/* ---- scalar pieces (unit-level parity) ---- */
void orc_box_create(int64_t n, const double* x, const double* y, const double* z,
                    int32_t force_cubic, double box9[9] /* min3, max3, size3 */);
void orc_compute_keys(int64_t n, const double* x, const double* y, const double* z,
                      const double boxmin[3], const double boxsize[3], int32_t curve,
                      int64_t* keys);
void orc_key_to_coord(int64_t key, const double boxmin[3], const double boxsize[3],
                      int32_t curve, double xout[3]);
/* In-place MSD radix sort of (key, index) pairs, reference sort order. */
void orc_sort_radix(int64_t n, int64_t* keys, int64_t* idx);
void orc_multipole_from_particle(const double pos[3], double q, double mp[15]);
void orc_shift_multipoles_up(double parent[15], const double* children, int32_t nchild);
void orc_force_leaf(const double node[15], const double delta[3], double dist2,
                    double e[3], double* phi);
void orc_force_twig(const double node[15], const double delta[3], double dist2,
                    double e[3], double* phi);
/* pepc-mini's portable generator; returns n draws after seeding with iseed
 * (iseed < 0: continue the default sequence from idum = -1). */
void orc_par_rand(int32_t iseed, int64_t n, double* out);

/* ---- whole-path context ---- */
typedef struct orc_ctx orc_ctx;
orc_ctx* orc_create(const orc_params* p);
void orc_destroy(orc_ctx* c);
/* grow: sorts, fixes duplicate keys, builds the tree and the moments.
 * Outputs in key order: keys, perm (0-based, sorted -> original), coordinates
 * (rewritten only for particles whose key was shifted), charges.
 * Returns 0, or a negative error code (-1 bad arg, -2 maxlevel/unsplittable). */
int orc_grow_tree(orc_ctx* c, int64_t n, const double* x, const double* y, const double* z,
                  const double* q, int64_t* key_out, int64_t* perm_out,
                  double* x_out, double* y_out, double* z_out, double* q_out);
/* traverse: accumulates (+=) e, pot and work onto nt targets.  tkeys may be
 * NULL (unkeyed targets: one tile each in the simple walk).
 * Returns 0 or -3 if a target did not see every leaf (walk incomplete). */
int orc_traverse_tree(orc_ctx* c, int64_t nt, const double* tx, const double* ty,
                      const double* tz, const int64_t* tkeys, double* ex, double* ey,
                      double* ez, double* pot, double* work);
/* number of nodes, leaves, twigs and the tree export (node order = the
 * reference's insertion order, module_tree_grow.f90:623-696, 0-based links). */
int64_t orc_num_nodes(const orc_ctx* c);
void orc_tree_export(const orc_ctx* c, int64_t* key, int32_t* level, int64_t* leaves,
                     int64_t* descendants, int64_t* parent, int64_t* first_child,
                     int64_t* next_sibling, double* moments15);
void orc_box(const orc_ctx* c, double box9[9]);
/* counters of the last traverse: interactions, mac evaluations */
void orc_counters(const orc_ctx* c, int64_t out[2]);
/* FP64 direct sum on the grown particles (module_directsum.f90:34-172):
 * targets are indices into the key-ordered particle array; includes the
 * mirror boxes and, if periodic with far field, the lattice term. */
int orc_direct(orc_ctx* c, int64_t ntest, const int64_t* tidx, double* ex, double* ey,
               double* ez, double* pot);
/* adjoint of the per-target walk with fixed interaction lists: dL/dq, dL/dx
 * of the grown particles (original order) for given dL/dE (gex..) and dL/dphi
 * at nt targets; with a periodic far field the lattice term's adjoint is added */
int orc_traverse_adjoint(orc_ctx* c, int64_t nt, const double* tx, const double* ty,
                         const double* tz, const double* gex, const double* gey,
                         const double* gez, const double* gphi, double* dLdq, double* dLdx,
                         double* dLdy, double* dLdz);
/* the same gradient by FP64 direct summation (no tree) */
int orc_direct_adjoint(orc_ctx* c, int64_t nt, const double* tx, const double* ty,
                       const double* tz, const double* gex, const double* gey, const double* gez,
                       const double* gphi, double* dLdq, double* dLdx, double* dLdy, double* dLdz);
/* install lattice coefficients (861 complex as interleaved re, im) before grow */
int orc_set_lattice_coefficients(orc_ctx* c, const double* re_im);
/* periodic lattice term alone for arbitrary positions (fmm_sum_lattice_force) */
int orc_lattice(orc_ctx* c, int64_t nt, const double* tx, const double* ty, const double* tz,
                double* ex, double* ey, double* ez, double* pot);

/* ---- the frontend's time step around the path (pepc-mini, module_helper.f90) ---- */
/* push_particles (:205-222): v += dt q/m E, then x += dt v */
void orc_push_particles(int64_t n, double dt, const double* q, const double* m, const double* ex,
                        const double* ey, const double* ez, double* vx, double* vy, double* vz,
                        double* x, double* y, double* z);
/* apply_external_field (:321-334): E_z += ez_ext, pot -= z ez_ext */
void orc_apply_external_field(int64_t n, double ez_ext, const double* z, double* ez, double* pot);
/* constrain_periodic (module_mirror_boxes.f90:177-218) with the parameters' lattice */
void orc_constrain_periodic(const orc_params* p, int64_t n, double* x, double* y, double* z);

#ifdef __cplusplus
}
#endif
#endif
