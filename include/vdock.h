/*
 * vdock -- B200-native Vina-style docking hot path, C ABI.
 *
 * Replaces the two host entry points of HPCLab-933/Vina-CUDA
 * (Vina-CUDA_v1.1):
 *   kernel_grid  (inc/cuda/kernel1.cuh:30-40, def kernel1.cu:202)  -> vd_build_grids
 *   kernel_monte (inc/cuda/kernel2.cuh:25-37, def kernel2.cu:566)  -> vd_dock / vd_dock_plain
 * and the host packing around them in lib/main_procedure_cu.cpp:131-1006.
 *
 * Conventions (all entry points):
 *   - plain C types only; host pointers unless a name ends in _device;
 *   - every call returns vd_status; vd_last_error() gives a message for the
 *     calling thread's last failure;
 *   - a context owns one CUDA device, its stream and all device buffers;
 *     calls on one context must not run concurrently (thread-compatible,
 *     not thread-safe per context);
 *   - calls are synchronous with respect to the host buffers they take.
 *
 * Pose layout ("conf", cf. output_type_cl, inc/kernel2.h:118-127):
 *   position[3], quaternion[4] (w,x,y,z), torsions[ntors]    stride 7+ntors
 * Gradient layout (cf. change_cl, inc/kernel2.h:129-136):
 *   force[3], torque[3], d/dtorsion[ntors]                    stride 6+ntors
 */
#ifndef VDOCK_H
#define VDOCK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    VD_OK = 0,
    VD_ERR_CUDA = 1,      /* a CUDA runtime call failed                        */
    VD_ERR_CAPACITY = 2,  /* input exceeds a compiled limit (atoms, torsions)  */
    VD_ERR_ARG = 3,       /* invalid argument or call order                    */
    VD_ERR_TIMEOUT = 4,   /* reserved: every device loop here is bounded by its
                             inputs and no kernel waits on another, so no call
                             returns it today                                 */
    VD_ERR_PARSE = 5,     /* malformed PDBQT / config input                    */
    VD_ERR_NOMEM = 6      /* device out of memory or the context's cap hit
                             (vd_set_memory_cap); the context stays usable     */
} vd_status;

#define VD_MAX_ATOMS 128      /* heavy atoms per ligand (inc/kernel2.h:36)      */
#define VD_MAX_TORS 48        /* torsions per ligand   (inc/kernel2.h:37)       */
#define VD_MAX_PAIRS 4096     /* intra-ligand pairs (reference: 2048)           */
#define VD_MAX_MODES 20       /* poses kept per ligand (main.cpp:394)           */
#define VD_XS_TYPES 17

typedef struct vd_ctx vd_ctx;

/* Ligand topology.  Atoms are grouped contiguously by rigid body and rigid
 * bodies are numbered in depth-first pre-order (body k>0 carries torsion k-1),
 * the order lib/parse_pdbqt.cpp:342-401 produces.  Atoms with xs < 0
 * (hydrogens) move with their body but carry no energy. */
typedef struct {
    int32_t n_atoms, n_nodes, n_pairs;
    const double*  xyz;              /* [n_atoms*3] input conformation             */
    const int32_t* xs;               /* [n_atoms] XS type 0..16 or -1              */
    const int32_t* el;               /* [n_atoms] element (0 = H)                  */
    const int32_t* atom_node;        /* [n_atoms] rigid body of each atom          */
    const int32_t* node_parent;      /* [n_nodes] parent body, -1 for the root     */
    const int32_t* node_origin_atom; /* [n_nodes] atom at the body's origin        */
    const int32_t* node_axis_atom;   /* [n_nodes] parent-side atom of the rotatable
                                        bond, -1 for the root                      */
    const int32_t* pairs;            /* [n_pairs*2] intra pairs (model.cpp:875-900) */
    double num_tors;                 /* N_tors of terms.cpp:97-128                 */
} vd_ligand_desc;

typedef struct {
    double v_intra;   /* curl cap of intra pairs  (v[0], model.cpp:1330)       */
    double v_inter;   /* curl cap of grid term    (v[1])                       */
    double slope;     /* out-of-box penalty slope (main.cpp:400: 1e6)          */
} vd_eval_params;

typedef struct {
    uint32_t seed;
    int32_t  n_chains;        /* MC chains per ligand (--thread)               */
    int32_t  search_depth;    /* MC steps per chain; 0 = main.cpp:354-391 rule,
                                 < 0 = none (chains return their initial pose) */
    int32_t  max_bfgs_steps;  /* 0 = (30 + atoms)/3 (main.cpp:386)             */
                              /* (25 + atoms)/3 with dense_bfgs             */
    int32_t  num_modes;       /* modes returned (<= VD_MAX_MODES)              */
    double   energy_range;    /* kcal/mol window above the best mode           */
    double   hunt_cap[3];     /* (10,10,10), main.cpp:395                      */
    double   temperature;     /* 1.2                                           */
    double   amplitude;       /* mutation amplitude 2 (monte_carlo.h:71)       */
    double   min_rmsd;        /* cluster radius 1.0                            */
    int32_t  refine;          /* 1 = refine + rescore on the GPU (main.cpp:434)*/
    int32_t  launch_shape;    /* docking kernel shape: 0 = autotuned per
                                 workload (among 1, 4, 5), 1/2/3/4/5 =
                                 64/48/40/80/128 registers per thread
                                 (8/10/12/6/4 blocks of 4 chains per SM);
                                 results do not depend on it                */
    int32_t  dense_bfgs;      /* local search of the Monte-Carlo steps:
                                 0 = RILC-BFGS (--rilc_bfgs 1, default,
                                 quasi_newton.cuh:2172-2389); 1 = dense BFGS
                                 (--rilc_bfgs 0, kernel2.cu:427-563): heuristic
                                 depth x 2.4 and (25 + atoms)/3 steps,
                                 main.cpp:367-389                           */
    int32_t  visited_history; /* 1 = QuickVina2-CUDA's visited history
                                 (QuickVina2-CUDA/inc/cuda/visited.cuh:48-227,
                                 quasi_newton.cuh:1937-1943), RILC-BFGS only:
                                 its novelty check returns false on every
                                 path, so each chain runs its first
                                 10 x (6 + ntors) local optimisations and
                                 keeps every later candidate unoptimised at
                                 its entry energy; 0 = off (Vina-CUDA)       */
} vd_search_params;

typedef struct {
    int32_t n_modes;
    int32_t ntors;
    float   energy[VD_MAX_MODES];          /* final score, ascending             */
    float   rmsd_lb[VD_MAX_MODES];         /* to mode 1 (model.cpp:1485-1507)    */
    float   rmsd_ub[VD_MAX_MODES];
    float   pose[VD_MAX_MODES][7 + VD_MAX_TORS];
    int64_t bfgs_evals;                    /* Monte-Carlo search energy+gradient
                                              evaluations of this ligand         */
} vd_dock_result;

typedef struct {
    int64_t bfgs_evals;          /* since the context was created               */
    double  grid_ms;             /* last vd_build_grids kernel time             */
    double  dock_ms;             /* last docking kernel time                    */
    double  post_ms;             /* last cluster+refine+rescore kernels time    */
    int32_t dock_warps_per_block;/* chains per block of the last docking launch  */
    int32_t dock_blocks;
    int32_t dock_shape;          /* launch_shape of the last docking launch (1-5) */
    int32_t grid_shape;          /* grid tile of the last build: 1 = 16x8x8 points
                                    per 256 threads, 2 = 16x8x4 per 128         */
    int64_t graph_launches;      /* batched pipelines submitted as a CUDA graph */
    int64_t graph_instantiations;/* executables built (the rest were updated in place) */
    double  scoring_ms;          /* wall time of the last vd_set_scoring(_device) */
    int64_t device_bytes;        /* device memory the context holds for maps, tables,
                                    ligands, receptor cells and scratch           */
    double  pair_force_scale;    /* fixed-point units per kcal/mol/A in which the
                                    kernels sum intra-pair forces (a power of two
                                    set from the current tables; 2^19 by default) */
    double  cells_ms;            /* last vd_build_grids: time to lay the maps out as
                                    32-byte trilinear corner cells for the
                                    evaluation kernels (0 when the box is too
                                    large for them and the kernels read the maps) */
    int64_t ligand_bytes;        /* device blobs of all ligands added since the
                                    last vd_clear_ligands (what the ligand uploads
                                    copy to the GPU)                            */
} vd_stats;

/* ---- context ------------------------------------------------------------ */
vd_status vd_create(vd_ctx** out, int device);
vd_status vd_destroy(vd_ctx* ctx);
const char* vd_last_error(void);
vd_status vd_get_stats(vd_ctx* ctx, vd_stats* out);
/* Caps the device memory the context may hold (bytes; 0 = no cap, the
 * default).  A call that would allocate past it -- or that finds the device
 * out of memory -- fails with VD_ERR_NOMEM and leaves the context usable:
 * raise the cap (or free work) and call again.  No reference counterpart
 * (the reference sizes its buffers statically, kernel2.h:46-52). */
vd_status vd_set_memory_cap(vd_ctx* ctx, int64_t bytes);

/* ---- scoring, receptor, box (main.cpp:337-345, 856-876) ------------------ */
/* weights: gauss1, gauss2, repulsion, hydrophobic, hydrogen, and the internal
 * rotor weight 5*w_rot/0.1-1 (main.cpp:862). */
vd_status vd_set_scoring(vd_ctx* ctx, const double weights[6]);
/* Same, with the tables built on the GPU (one thread per table entry) for
 * weight sweeps: the host build takes milliseconds per weight set.  The
 * arithmetic and order are the host's; only exp() may differ by an ulp, so
 * tables agree with vd_set_scoring's to ~1e-15 relative (precalculate.h:255-283
 * on the device; no reference counterpart as an entry point). */
vd_status vd_set_scoring_device(vd_ctx* ctx, const double weights[6]);
vd_status vd_set_receptor(vd_ctx* ctx, int32_t n_atoms, const double* xyz, const int32_t* xs);
vd_status vd_set_box(vd_ctx* ctx, const double center[3], const double size[3]);
vd_status vd_grid_dims(vd_ctx* ctx, int32_t npts[3], double begin[3], double end[3]);

/* ---- grid maps: replaces kernel_grid (kernel1.cu:202-249) ----------------- */
/* Builds one FP32 map per listed XS type over the box; maps stay on device. */
vd_status vd_build_grids(vd_ctx* ctx, const int32_t* xs_types, int32_t n_types);
/* Grid tile of later builds: 0 = autotuned (the first build of each box size
 * times both tiles), 1 = 16x8x8 points per 256 threads, 2 = 16x8x4 per 128.
 * The maps are bit-identical for every tile. */
vd_status vd_set_grid_shape(vd_ctx* ctx, int32_t shape);
/* Copies one map to the host, x fastest: out[x + nx*(y + ny*z)]. */
vd_status vd_get_grid(vd_ctx* ctx, int32_t xs_type, float* out);

/* ---- ligands -------------------------------------------------------------- */
vd_status vd_add_ligand(vd_ctx* ctx, const vd_ligand_desc* lig, int32_t* lig_id);
/* n ligands at once (the per-ligand packing of main_procedure_cu.cpp:550-846
 * for a whole list): the blobs, pair segments and search schedules are built
 * on up to 32 host threads, then appended in list order, so lig_ids and
 * every later result equal n vd_add_ligand calls.  If a descriptor is
 * invalid, none is added and the error names its index. */
vd_status vd_add_ligands(vd_ctx* ctx, const vd_ligand_desc* ligs, int32_t n, int32_t* lig_ids);
vd_status vd_ligand_info(vd_ctx* ctx, int32_t lig_id, int32_t* n_heavy, int32_t* ntors,
                         int32_t* n_pairs);
vd_status vd_clear_ligands(vd_ctx* ctx);

/* ---- pose batches: forward energy and adjoint (model.cpp:1324-1333) ------- */
vd_status vd_energy(vd_ctx* ctx, int32_t lig_id, int32_t n_poses, const float* poses,
                    const vd_eval_params* p, float* e_out);
vd_status vd_energy_grad(vd_ctx* ctx, int32_t lig_id, int32_t n_poses, const float* poses,
                         const vd_eval_params* p, float* e_out, float* g_out);
/* Same on device buffers already resident, asynchronous on `stream` (a
 * cudaStream_t; NULL is the CUDA default stream, as for a kernel launch), so
 * a caller orders it with its own work by passing its stream (e.g. torch's
 * current stream).  Ligand and map uploads made by earlier calls have
 * completed before these return. */
vd_status vd_energy_grad_device(vd_ctx* ctx, int32_t lig_id, int32_t n_poses,
                                const float* poses_device, const vd_eval_params* p,
                                float* e_device, float* g_device, void* stream);
vd_status vd_energy_device(vd_ctx* ctx, int32_t lig_id, int32_t n_poses, const float* poses_device,
                           const vd_eval_params* p, float* e_device, void* stream);
/* Heavy-atom coordinates of poses (forward kinematics only): [n][n_heavy][3]. */
vd_status vd_pose_coords(vd_ctx* ctx, int32_t lig_id, int32_t n_poses, const float* poses,
                         float* xyz_out);

/* ---- local optimisation (quasi_newton.cuh:2172-2389, 1710-1806) ------------ */
/* One RILC-BFGS run per pose on the cached grid; poses are updated in place. */
vd_status vd_local_opt(vd_ctx* ctx, int32_t lig_id, int32_t n_poses, float* poses,
                       const vd_eval_params* p, int32_t max_steps, float* e_out,
                       int64_t* evals);

/* ---- Monte-Carlo search: replaces kernel_monte (kernel2.cu:566-628) -------- */
/* Raw per-chain best poses and energies of one ligand (one launch).  poses:
 * [n_chains][7+ntors], e: [n_chains].  Chains use Philox streams keyed by
 * (seed, lig_id, chain), so the batched and plain forms give equal chains. */
vd_status vd_mc_chains(vd_ctx* ctx, int32_t lig_id, const vd_search_params* sp,
                       float* poses_out, float* e_out, int64_t* evals);
/* Same chains as vd_mc_chains (same kernel and random streams) for callers
 * that cannot allocate device memory when they dock: hosts that reserve
 * their whole device-memory budget up front (a pool owning every free byte,
 * a service that must not grow its footprint on a shared GPU) and
 * latency-sensitive hosts that cannot take the device-wide synchronisation
 * an allocation may imply.  No counterpart in the reference.
 * It allocates nothing: parameters, counters and results pass through a
 * static device array of VD_NOALLOC_SCRATCH_BYTES (4 MiB) that every GPU
 * loading the library holds until exit; calls needing more are rejected
 * (VD_ERR_CAPACITY).  All calls on a device share that array and it keeps
 * the last call's contents, so calls whose GPU work overlaps race: serialise
 * them.  Ligands must already be on the device (one allocating call after
 * vd_add_ligand).  The first call on a device looks up the array's address
 * once (set-up); make it before any stream capture.  sp->launch_shape is not
 * read: the kernel runs at the 64-register shape (chains are identical at
 * every shape).  Evaluations are added to vd_stats.bfgs_evals; dock_ms is
 * not updated. */
#define VD_NOALLOC_SCRATCH_BYTES (4u << 20)
vd_status vd_mc_chains_noalloc(vd_ctx* ctx, int32_t lig_id, const vd_search_params* sp,
                               float* poses_out, float* e_out, int64_t* evals);
/* Plain drop-in form: one ligand per launch, then clustering, GPU refinement
 * and rescoring (main.cpp:423-489). */
vd_status vd_dock_plain(vd_ctx* ctx, int32_t lig_id, const vd_search_params* sp,
                        vd_dock_result* out);
/* Batched form: all chains of all listed ligands in one persistent launch that
 * pulls (ligand, chain) items from a device queue; post-processing batched. */
vd_status vd_dock_batched(vd_ctx* ctx, const int32_t* lig_ids, int32_t n_ligs,
                          const vd_search_params* sp, vd_dock_result* out);

/* ---- refinement / rescoring on the direct-sum score (non_cache.cpp) -------- */
/* refine_structure (main.cpp:139-157): dense BFGS with the slope ramp. */
vd_status vd_refine(vd_ctx* ctx, int32_t lig_id, int32_t n_poses, float* poses,
                    int32_t max_steps, float* e_out);
/* eval_adjusted (model.cpp:1428-1431) with intra energy of pose 0 as the
 * reference, plus the intramolecular energies themselves. */
vd_status vd_score(vd_ctx* ctx, int32_t lig_id, int32_t n_poses, const float* poses,
                   float* adjusted_out, float* intra_out);

/* RMSD lower / upper bounds of each pose's heavy atoms to pose 0
 * (model.cpp:1485-1523, the rmsd l.b. / u.b. of the REMARK VINA RESULT lines,
 * main.cpp:159-170); the same device code as vd_dock_*'s mode output. */
vd_status vd_rmsd_bounds(vd_ctx* ctx, int32_t lig_id, int32_t n_poses, const float* poses,
                         float* lb_out, float* ub_out);

/* ---- host helpers (no GPU work) --------------------------------------------- */
/* Pair tables built by vd_set_scoring: fast[153][2051], smooth e / dor. */
vd_status vd_get_tables(vd_ctx* ctx, double* fast, double* smooth_e, double* smooth_dor);
/* PDBQT ingestion (lib/parse_pdbqt.cpp, lib/model.cpp typing).  Returned
 * arrays are owned by the handle and live until vd_pdbqt_free. */
typedef struct vd_pdbqt vd_pdbqt;
vd_status vd_pdbqt_ligand(const char* text, vd_pdbqt** out, vd_ligand_desc* desc);
vd_status vd_pdbqt_receptor(const char* text, vd_pdbqt** out, int32_t* n_atoms,
                            const double** xyz, const int32_t** xs);
/* Writes a docked model: the input ligand text with coordinates replaced
 * (model.cpp:1088-1116); xyz_all holds every ligand atom [n_atoms][3]. */
vd_status vd_pdbqt_write_model(vd_pdbqt* lig, const double* xyz_all, char* buf, int64_t buf_size,
                               int64_t* written);
vd_status vd_pdbqt_free(vd_pdbqt* h);
/* All-atom coordinates (hydrogens included) for a pose, on the host, from the
 * descriptor (tree.h:395-400 set_conf), for writing output files. */
vd_status vd_conf_to_coords(const vd_ligand_desc* lig, const float* pose, double* xyz_all);

#ifdef __cplusplus
}
#endif
#endif /* VDOCK_H */
