/*
 * pepcg.h -- C ABI of libpepcg, a B200-native (sm_100a) implementation of
 * PEPC's Barnes-Hut tree-code force evaluation (Coulomb backend).
 *
 * The library replaces, for one MPI rank on one GPU, the reference's
 *   module_pepc::pepc_grow_tree      (src/treecode/lpepcsrc/module_pepc.f90:435-446)
 *   module_pepc::pepc_traverse_tree  (src/treecode/lpepcsrc/module_pepc.f90:459-468)
 *   module_pepc::pepc_timber_tree    (src/treecode/lpepcsrc/module_pepc.f90:538)
 * and the Coulomb interaction-backend API
 *   (src/interaction_specific/coulomb/module_interaction_specific.f90:46-60).
 *
 * Conventions
 *  - Every function returns an int status: PEPCG_OK (0) or a PEPCG_ERR_* code;
 *    pepcg_last_error() returns a human-readable message for the last error.
 *  - Plain pointers and sizes only.  "Host" entry points take host memory and
 *    do their own transfers; "_device" entry points take device pointers
 *    (cudaMalloc'd, on the context's device) and never synchronise the host
 *    beyond what their return status requires.
 *  - A context is used by one host thread at a time; calls are ordered on the
 *    context's CUDA stream.  The caller owns all arrays it passes; the context
 *    owns its device tree buffers from grow until timber/destroy.
 *  - Results of the traversal are ACCUMULATED (+=) into the caller's arrays,
 *    exactly like particle%results in the reference, which the frontend clears
 *    (pepc_particleresults_clear) before growing.
 */
#ifndef PEPCG_H
#define PEPCG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define PEPCG_OK 0
#define PEPCG_ERR_BAD_ARG 1         /* invalid argument or parameter */
#define PEPCG_ERR_CUDA 2            /* CUDA runtime error (message has the detail) */
#define PEPCG_ERR_OOM 3             /* device allocation failed */
#define PEPCG_ERR_NODE_POOL 4       /* tree larger than the node pool */
#define PEPCG_ERR_MAXLEVEL 5        /* unsplittable keys (module_tree_grow.f90:671-675) */
#define PEPCG_ERR_INCOMPLETE_WALK 6 /* a target did not see all N leaves
                                       (module_tree_walk_pthreads.f90:452-457) */
#define PEPCG_ERR_TIMEOUT 7         /* a bounded device-side wait gave up */
#define PEPCG_ERR_NO_TREE 8         /* traverse/stats called without a grown tree */
#define PEPCG_ERR_UNSUPPORTED 9     /* parameter combination not implemented */
#define PEPCG_WARN_NOT_NEUTRAL 100  /* periodic box not neutral; monopole removed
                                       (module_fmm_framework.f90:570-573).  A warning:
                                       the call completed. */

/* ---- parameter enums ---- */
#define PEPCG_CURVE_HILBERT 0 /* the reference's curve (module_spacefilling.f90:380-440) */
#define PEPCG_CURVE_MORTON 1  /* 3D Z-order; not in the reference for idim = 3 */

#define PEPCG_PRECISION_PLAIN 0 /* FP64 throughout: the drop-in */
#define PEPCG_PRECISION_MIXED 1 /* FP64 offsets + FP32 interactions + FP64 sums */
#define PEPCG_PRECISION_MIXED_STRICT 2 /* the mixed form with every interaction offset the
                                          target minus the node centre in FP64, rounded
                                          once, Kahan-compensated FP32 sums, and the FP64
                                          group walk's MAC decisions; GROUP walk with
                                          64-target buckets */

#define PEPCG_WALK_PER_TARGET 0 /* module_tree_walk_pthreads semantics (pepc-mini) */
#define PEPCG_WALK_PER_TILE 1   /* module_tree_walk_simple semantics (pepc-essential) */
#define PEPCG_WALK_GROUP 2      /* warp-bucket group walk: buckets of group_size key-
                                   consecutive targets, node lists batched through shared
                                   memory */

/*
 * Parameters: the /libpepc/ and /calc_force_coulomb/ namelist variables that
 * the Coulomb tree code reads (module_libpepc_main.f90:44,
 * coulomb/module_interaction_specific.f90:35-43, module_mirror_boxes.f90:30-38,
 * module_fmm_framework.f90:49), plus the GPU walk selection.
 */
typedef struct pepcg_params {
  double theta2;                 /* square of the BH opening angle [0.36] */
  double eps2;                   /* Plummer softening squared [0.0] */
  int32_t force_law;             /* 3 3D Coulomb, 2 2D Coulomb, 4 Lennard-Jones, 5 Kelbg
                                    (2, 4, 5: plain form) [3] */
  int32_t mac_select;            /* 0 Barnes-Hut, 1 Bmax, other > 0: no acceptance (N^2) [0] */
  int32_t curve;                 /* PEPCG_CURVE_* [HILBERT] */
  int32_t precision;             /* PEPCG_PRECISION_* [PLAIN] */
  int32_t walk;                  /* PEPCG_WALK_* [PER_TARGET] */
  int32_t tile_size;             /* PER_TILE: max targets per tile, 1..32 [16] */
  int32_t force_cubic_domain;    /* module_box.f90:28 [0] */
  int32_t periodicity[3];        /* module_mirror_boxes.f90:37 [0,0,0] */
  int32_t mirror_box_layers;     /* module_mirror_boxes.f90:38 [1] */
  int32_t include_far_field_if_periodic; /* specific.f90:37 [1] */
  int32_t fmm_extrinsic_correction;      /* 0 none, 1 Redlack, 2 fictitious charges [2] */
  double t_lattice_1[3];         /* lattice basis [1,0,0] */
  double t_lattice_2[3];         /* [0,1,0] */
  double t_lattice_3[3];         /* [0,0,1] */
  double lattice_origin[3];      /* [0,0,0] */
  int32_t device;                /* CUDA device ordinal [0] */
  int32_t overwrite_results;     /* pepcg_traverse_tree: 0 = add to ex..work (+=, like
                                    particle%results) [0]; 1 = overwrite them (the frontend's
                                    results clear and the traverse in one call, with no
                                    upload of the old values) */
  double kelbg_invsqrttemp;      /* force_law 5: 1/sqrt(temperature) (specific.f90:40) [0] */
  int32_t group_size;            /* GROUP walk: targets per bucket, 32 or 64; 0 = 64 for the
                                    mixed walk and 32 for the plain walk [0].  The adjoint
                                    supports both. */
  int32_t reserved0;             /* zero */
  double spatial_interaction_cutoff[3]; /* module_mirror_boxes.f90:52: a node whose offset
                                    from the target has any |component| >= the cutoff is
                                    skipped (module_tree_walk_pthreads.f90:622,639;
                                    module_tree_walk_simple.f90:330,377); plain walks and
                                    their adjoint only, >= 0 [DBL_MAX each: no cutoff] */
  int32_t reserved[4];           /* zero */
} pepcg_params;

/* Statistics of the last grow/traverse (module_tree.f90:622-699,
 * module_tree_walk_pthreads.f90:149-201) and per-phase device times. */
typedef struct pepcg_stats {
  int64_t npart;
  int64_t nleaf;
  int64_t ntwig;
  int64_t max_level;
  int64_t dup_count;            /* adjacent equal keys found before the fix */
  int64_t interactions;         /* leaf + twig interactions of the last traverse */
  int64_t leaf_interactions;
  int64_t twig_interactions;
  int64_t mac_evaluations;
  double t_keys_ms, t_sort_ms, t_tree_ms, t_upward_ms, t_walk_ms, t_lattice_ms;
  double box[9];                /* boxmin(3), boxmax(3), boxsize(3) */
} pepcg_stats;

void pepcg_params_default(pepcg_params* p);
int pepcg_create(void** ctx, const pepcg_params* p);
int pepcg_destroy(void* ctx);
const char* pepcg_last_error(const void* ctx);
/* change theta2 / eps2 / precision / walk between traversals */
int pepcg_set_params(void* ctx, const pepcg_params* p);

/*
 * pepcg_grow_tree -- replaces pepc_grow_tree (module_pepc.f90:435-446) ->
 * libpepc_grow_tree (module_libpepc_main.f90:105-124) -> tree_grow
 * (module_tree_grow.f90:37-138) at one rank: bounding box, keys, local sort,
 * duplicate-key fix (module_domains.f90:158-319), octree and multipoles, and
 * the periodic lattice preparation (calc_force_after_grow).
 * Inputs: n >= 2 particles (x, y, z, q), host arrays.
 * Outputs (each may be NULL), all in key order:
 *   key_out  particle keys (kind_key)
 *   perm_out 0-based original index of each key-ordered particle; the caller
 *            reorders its particle records with it (particles stay in key
 *            order across steps, as in pepc-mini)
 *   x_out.. coordinates in key order (rewritten by key_to_coord only for
 *            particles whose duplicate key was shifted)
 */
int pepcg_grow_tree(void* ctx, int64_t n, const double* x, const double* y, const double* z,
                    const double* q, int64_t* key_out, int64_t* perm_out, double* x_out,
                    double* y_out, double* z_out);
/* Same with device-resident inputs; the key-ordered state stays on the device. */
int pepcg_grow_tree_device(void* ctx, int64_t n, const double* d_x, const double* d_y,
                           const double* d_z, const double* d_q);
/* Copy the key-ordered particle state of the grown tree (device pointers). */
int pepcg_get_particles_device(void* ctx, int64_t* d_key, int64_t* d_perm, double* d_x,
                               double* d_y, double* d_z, double* d_q);

/*
 * pepcg_traverse_tree -- replaces pepc_traverse_tree (module_pepc.f90:459-468)
 * -> libpepc_traverse_tree (module_libpepc_main.f90:161-200): one walk per
 * mirror box (central box last), then the per-particle lattice term
 * (calc_force_per_particle, coulomb/module_interaction_specific.f90:393-427).
 * Targets: nt positions (host).  tkeys: the targets' keys when they are keyed
 * (the grown particles), or NULL (each target is its own tile in PER_TILE).
 * Accumulates (+=) ex, ey, ez, pot and work (+1 per interaction).
 */
int pepcg_traverse_tree(void* ctx, int64_t nt, const double* tx, const double* ty,
                        const double* tz, const int64_t* tkeys, double* ex, double* ey,
                        double* ez, double* pot, double* work);
/* Same with device arrays. */
int pepcg_traverse_tree_device(void* ctx, int64_t nt, const double* d_tx, const double* d_ty,
                               const double* d_tz, const int64_t* d_tkeys, double* d_ex,
                               double* d_ey, double* d_ez, double* d_pot, double* d_work);
/* Targets = the grown particles themselves, in key order (device results). */
int pepcg_traverse_self_device(void* ctx, double* d_ex, double* d_ey, double* d_ez,
                               double* d_pot, double* d_work);

/*
 * pepcg_traverse_adjoint -- the adjoint of pepcg_traverse_tree (no reference
 * counterpart; the reference has no differentiation).  Given dL/dE (three
 * arrays) and dL/dphi at nt targets, returns dL/dq and dL/dx, dL/dy, dL/dz of
 * the grown particles in the caller's ORIGINAL order (overwrites; arrays of
 * length npart).  The interaction lists are recomputed with the context's walk
 * semantics and held fixed (MAC decisions and keys are piecewise constant).
 * The plain walks' adjoints are FP64.  With the mixed GROUP walk and 64-target
 * buckets (the mixed default) the adjoint runs on that walk's own FP32 lists,
 * evaluates its terms in FP32 on the group-centred offsets and sums them in
 * FP64 across buckets, like the forward; the other mixed walks take the FP64
 * adjoint of their semantics.  Force laws 3 (3D Coulomb, closed forms), 2 (2D
 * Coulomb) and 4 (Lennard-Jones): the last two differentiate the forward
 * kernels themselves (forward-mode dual numbers for the offset, unit moments
 * for the charge and moments), FP64 walks only, as the forward.  Law 5
 * (Kelbg) returns PEPCG_ERR_UNSUPPORTED: its leaf kernel needs each target's
 * own charge, which the adjoint's targets do not carry.  With periodic
 * boundaries the mirror boxes'
 * terms are in the walk's adjoint, and the FMM far-lattice term's adjoint
 * (FP64, every fmm_extrinsic_correction) is added: the transpose of the
 * lattice force and of the central box's multipole expansion, through the
 * fictitious charges or Redlack terms to the particles.
 */
int pepcg_traverse_adjoint(void* ctx, int64_t nt, const double* tx, const double* ty,
                           const double* tz, const double* dLdEx, const double* dLdEy,
                           const double* dLdEz, const double* dLdphi, double* dLdq, double* dLdx,
                           double* dLdy, double* dLdz);
/* Same with device arrays. */
int pepcg_traverse_adjoint_device(void* ctx, int64_t nt, const double* d_tx, const double* d_ty,
                                  const double* d_tz, const double* d_gex, const double* d_gey,
                                  const double* d_gez, const double* d_gphi, double* d_dq,
                                  double* d_dx, double* d_dy, double* d_dz);

/*
 * The frontend's time step around the path, on device arrays and the
 * context's stream, so particles can stay on the GPU between steps.  These
 * replace loops of the pepc-mini frontend rather than library routines:
 *   pepcg_push_particles_device       push_particles (frontends/pepc-mini/
 *     module_helper.f90:205-222): v += dt q/m E, then x += dt v (in place);
 *   pepcg_apply_external_field_device apply_external_field (:321-334):
 *     E_z += ez_ext, pot -= z ez_ext (in place);
 *   pepcg_constrain_periodic_device   constrain_periodic (module_mirror_boxes.f90:
 *     177-218): positions wrapped into the context's lattice cell along its
 *     periodic directions (in place);
 *   pepcg_gather_device               out[i] = in[perm[i]] with the last grow's
 *     permutation (n of that grow), to carry per-particle state such as
 *     velocity or mass into key order as the reference's domain_decompose
 *     (module_domains.f90:158-319) moves whole particle records; in != out.
 * Results are the reference expressions in their order, bit for bit.
 */
int pepcg_push_particles_device(void* ctx, int64_t n, double dt, const double* d_q,
                                const double* d_m, const double* d_ex, const double* d_ey,
                                const double* d_ez, double* d_vx, double* d_vy, double* d_vz,
                                double* d_x, double* d_y, double* d_z);
int pepcg_apply_external_field_device(void* ctx, int64_t n, double ez_ext, const double* d_z,
                                      double* d_ez, double* d_pot);
int pepcg_constrain_periodic_device(void* ctx, int64_t n, double* d_x, double* d_y, double* d_z);
int pepcg_gather_device(void* ctx, const double* d_in, double* d_out);
/*
 * pepcg_potential_energy_device -- the potential energy of pepc-b's
 * diagnostics (potenergy, frontends/pepc-b/module_diagnostics.f90:227-263):
 * *epot = sum over the n particles of 0.5 q phi, accumulated in FP64 on the
 * device (block partials added in a fixed order, so the result does not vary
 * from run to run; the reference's sequential sum differs from it only by
 * rounding), so the potentials need not come back to the host.  d_q and d_pot
 * are device arrays in the same order; epot is a host pointer (the call waits
 * for the result).
 */
int pepcg_potential_energy_device(void* ctx, int64_t n, const double* d_q, const double* d_pot,
                                  double* epot);

/*
 * Sharding the targets of the grown particles over ranks (one GPU each, the
 * tree replicated), and the way back to the caller's order.  No reference
 * entry points: they stand for the MPI domain split of the particles
 * (module_domains.f90) and domain_restore (:372-408).
 *   pepcg_traverse_range_device  the fields on the grown particles [t0, t1) of
 *     the key order, written to arrays of length t1 - t0 (accumulates like
 *     pepcg_traverse_self_device); ranges that start at multiples of the group
 *     walk's bucket (64 covers both sizes) give exactly the single-call result
 *     in every walk mode;
 *   pepcg_restore_device         out[perm[i]] = in[i]: a key-ordered array back
 *     to the order of the last grow's input (in != out).
 */
int pepcg_traverse_range_device(void* ctx, int64_t t0, int64_t t1, double* d_ex, double* d_ey,
                                double* d_ez, double* d_pot, double* d_work);
int pepcg_restore_device(void* ctx, const double* d_in, double* d_out);

/* Launch all of this context's work on the caller's CUDA stream (a
 * cudaStream_t of the context's device), or on a private non-blocking stream
 * when NULL (so the legacy default stream is selected with cudaStreamLegacy).
 * Lets a caller that owns a stream (e.g. a framework's current stream) order
 * and time the library's kernels with its own events.  No reference
 * counterpart: the reference has no device streams. */
int pepcg_set_stream(void* ctx, void* stream);
/* Total number of kernels this library has launched in the process. */
long long pepcg_kernel_launches(void);

/*
 * pepcg_debug_fail_allocations -- allocation-failure injection for tests, in
 * the spirit of the reference's DEBUG_ERROR checks (module_debug.f90:167),
 * which abort the run; here the failing call returns a status instead.  After
 * `after` more successful device allocations by the library (in this
 * process), every further one fails as if the device had run out of memory,
 * so the call that needed it returns PEPCG_ERR_OOM and leaves its context
 * usable (a later call allocates again).  A negative value switches the
 * injection off, which is the default.  Host side only: nothing reaches the
 * device.
 */
void pepcg_debug_fail_allocations(int64_t after);

/* replaces pepc_timber_tree (module_pepc.f90:538 -> module_libpepc_main.f90:129-148) */
int pepcg_timber_tree(void* ctx);
int pepcg_stats_get(void* ctx, pepcg_stats* s);

/*
 * Tree export in the reference's node order (insertion order of
 * module_tree_grow.f90:623-696, 0-based indices, -1 = NODE_INVALID), for
 * parity checks and diagnostics.  Arrays of length pepcg_num_nodes(); any may
 * be NULL.  moments15: 15 doubles per node in t_tree_node_interaction_data
 * order (module_interaction_specific_types_XYZQVM.f90:47-57).
 */
int64_t pepcg_num_nodes(void* ctx);
int pepcg_tree_export(void* ctx, int64_t* key, int32_t* level, int64_t* leaves,
                      int64_t* descendants, int64_t* parent, int64_t* first_child,
                      int64_t* next_sibling, double* moments15);

/*
 * FP64 direct sum on sampled targets (module_directsum.f90:34-172): targets
 * are indices into the key-ordered particles; includes all mirror boxes with
 * the self term excluded in the central box, then the lattice term.
 * Overwrites (=) ex, ey, ez, pot (host arrays of length ntest).
 */
int pepcg_direct(void* ctx, int64_t ntest, const int64_t* tidx, double* ex, double* ey,
                 double* ez, double* pot);

/* Periodic far-lattice term alone (fmm_sum_lattice_force,
 * module_fmm_framework.f90:766-826) at nt positions; overwrites. */
int pepcg_lattice(void* ctx, int64_t nt, const double* tx, const double* ty, const double* tz,
                  double* ex, double* ey, double* ez, double* pot);
/* The same at one position, in the shape of fmm_sum_lattice_force(pos, e_lattice,
 * phi_lattice) (module_fmm_framework.f90:766-826), for shims that call it per
 * particle as calc_force_per_particle does (coulomb/module_interaction_specific.
 * f90:393-427).  Overwrites e[3] and *phi. */
int pepcg_lattice_force(void* ctx, const double pos[3], double e[3], double* phi);

/*
 * pepcg_sort_keys -- replaces the local key sort of domain_decompose
 * (module_domains.f90:182, slsort_keys -> sl_pepc/mpi_pepckeys.c:151-167 ->
 * pepckeys_sort_radix, sort_radix.c:122-151) at one rank: sorts n keys
 * (host arrays) and returns the sorted keys and the 0-based input index of
 * each sorted key (slsort_keys' indxl, minus one).  Keys are ordered as
 * unsigned 64-bit values, as the reference's radix sort orders them (PEPC's
 * keys are non-negative).  Equal keys come out in the order the reference's
 * in-place MSD radix sort leaves them, which is the order pepcg_grow_tree
 * gives to particles with equal keys.  Either output may be NULL.
 */
int pepcg_sort_keys(void* ctx, int64_t n, const int64_t* keys, int64_t* keys_out,
                    int64_t* perm_out);
/* Same with device arrays, on the context's stream. */
int pepcg_sort_keys_device(void* ctx, int64_t n, const int64_t* d_keys, int64_t* d_keys_out,
                           int64_t* d_perm_out);

/*
 * pepcg_sort_keys_noalloc -- sorts n 64-bit keys (ascending as unsigned
 * 64-bit values, so a negative key sorts after every non-negative one;
 * stable: equal keys keep their input order) and returns the sorted keys and
 * the 0-based input index of each sorted key, all device pointers, enqueued
 * on `stream` (a cudaStream_t of the current device, or NULL).  It allocates
 * nothing: for callers that cannot call cudaMalloc, its scratch is a static
 * device array of the library (about 24.3 MB per device, held until exit),
 * which limits n to 1,048,576; larger n returns PEPCG_ERR_BAD_ARG.  The first
 * call on a device looks up that array's address and keeps it for the life of
 * the process (make that call before any stream capture; a device reset
 * between calls is not supported); calls that overlap on the GPU race on the
 * shared array.  For distinct keys the order equals pepcg_grow_tree's and
 * pepcg_sort_keys'; equal keys keep their input order here, where those two
 * give the reference's order.
 * No counterpart in the reference.
 */
int pepcg_sort_keys_noalloc(int64_t n, const int64_t* d_keys_in, int64_t* d_keys_out,
                            int64_t* d_perm_out, void* stream);

/* ---- scalar backend entry points (evaluated by the same device code the
 * walk uses; one tiny launch per call, for shims and unit tests) ---- */
/* multipole_from_particle, coulomb/module_interaction_specific.f90:67-79 */
int pepcg_multipole_from_particle(const double pos[3], double q, double mp[15]);
/* shift_multipoles_up, coulomb/module_interaction_specific.f90:84-140 */
int pepcg_shift_multipoles_up(double parent[15], const double* children, int32_t nchild);
/* calc_force_per_interaction_with_leaf / _with_twig for force_law 3
 * (specific.f90:314-387 -> module_coulomb_kernels.f90:242-257 / :60-145);
 * dist2 is |delta|^2 and eps2 is added inside, like the reference wrappers. */
int pepcg_force_with_leaf(const double node[15], const double delta[3], double dist2,
                          double eps2, double e[3], double* phi);
int pepcg_force_with_twig(const double node[15], const double delta[3], double dist2,
                          double eps2, double e[3], double* phi);
/* mac (specific.f90:256-275), Barnes-Hut: theta2 * dist2 > boxlength2 */
int pepcg_mac(double theta2, double dist2, double boxlength2, int32_t* accept);

#ifdef __cplusplus
}
#endif
#endif /* PEPCG_H */
