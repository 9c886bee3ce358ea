/*
 * ORACLE -- test infrastructure only, never shipped or measured as the product.
 *
 * CPU double-precision restatement of the AutoDock-Vina scoring, grid,
 * kinematics, optimiser and search code that HPCLab-933/Vina-CUDA
 * (tree Vina-CUDA_v1.1) uses on its docking hot path.  Each function cites
 * the reference file:line it follows.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load liboracle.so.
 *
 * Parity status: the reference cannot be compiled here (its sources need the
 * Boost 1.77 headers, which are absent), so there is no oracle/_ref build.
 * The scoring function is pinned by a known-answer test that rescores the
 * docked poses the reference ships (REMARK VINA RESULT energies and RMSD
 * columns of Vina-CUDA_v1.1/docking_result/1u1b_docking_result.pdbqt and the
 * QuickVina-W-CUDA example outputs); the optimiser and search restatements
 * are unpinned (the reference records no seeds or trajectories).
 */
#ifndef VINA_ORACLE_H
#define VINA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_ctx or_ctx;

/* Ligand topology, identical in meaning to vd_ligand_desc (include/vdock.h). */
typedef struct {
    int32_t n_atoms, n_nodes, n_pairs;
    const double*  xyz;              /* [n_atoms*3] input conformation       */
    const int32_t* xs;               /* [n_atoms] XS type 0..16, -1 = none   */
    const int32_t* el;               /* [n_atoms] element type (EL_TYPE_*)   */
    const int32_t* atom_node;        /* [n_atoms] owning rigid body           */
    const int32_t* node_parent;      /* [n_nodes] -1 for the root             */
    const int32_t* node_origin_atom; /* [n_nodes]                             */
    const int32_t* node_axis_atom;   /* [n_nodes] parent-side atom, -1 root   */
    const int32_t* pairs;            /* [n_pairs*2] intra pairs (a,b)         */
    double num_tors;                 /* conf-independent N_tors               */
} or_ligand;

or_ctx* or_create(const double weights[6]);
void    or_destroy(or_ctx*);
/* Pair tables: type pair p (t1<=t2, p = t1 + t2*(t2+1)/2), index i < 2051. */
void    or_tables(or_ctx*, double* fast, double* smooth_e, double* smooth_dor);
int     or_set_receptor(or_ctx*, int n, const double* xyz, const int32_t* xs);
/* Grid dims exactly as main.cpp:864-876 (granularity 0.375). */
int     or_set_box(or_ctx*, const double center[3], const double size[3]);
void    or_grid_info(or_ctx*, int32_t npts[3], double begin[3], double end[3]);
int     or_build_grids(or_ctx*, const int32_t* types, int n_types);
int     or_get_grid(or_ctx*, int xs_type, double* out /* x fastest */);
int     or_add_ligand(or_ctx*, const or_ligand*);
int     or_ligand_ntors(or_ctx*, int lig);
/* 1 when the maps of every heavy-atom type of the ligand are built; the cached
 * evaluations below return NaN (or_mc_chains: -1) otherwise. */
int     or_maps_ready(or_ctx*, int lig);

/* conf layout: pos[3], quat[4] (w,x,y,z), torsions[ntors]
 * grad layout: force[3], torque[3], torsion grads[ntors]
 * v[3] = (intra cap, inter cap, other-pair cap) as in model.cpp:1324. */
/* Unweighted intermolecular terms (gauss1, gauss2, repulsion, hydrophobic,
 * hydrogen bond) of heavy-atom coordinates xyz, analytic (terms.cpp:385-446),
 * and the torsion normalisation x / (1 + w N_tors / 5) (everything.cpp:294-301). */
void    or_term_values_coords(or_ctx*, int lig, const double* xyz, double out[5]);
double  or_conf_independent(or_ctx*, int lig, double x);
double  or_eval_deriv(or_ctx*, int lig, const double* conf, const double v[3],
                      double slope, double* grad /* may be NULL */);
void    or_coords(or_ctx*, int lig, const double* conf, double* xyz_out /* all atoms */);
double  or_eval_intramolecular(or_ctx*, int lig, const double* conf, double v_intra);
double  or_nc_eval_deriv(or_ctx*, int lig, const double* conf, const double v[3],
                         double slope, double* grad);
double  or_eval_adjusted(or_ctx*, int lig, const double* conf, double intra_best);
double  or_eval_adjusted_coords(or_ctx*, int lig, const double* xyz_all, double intra_best);
double  or_intramolecular_coords(or_ctx*, int lig, const double* xyz_all);
double  or_rmsd_upper(or_ctx*, int lig, const double* xyz_a, const double* xyz_b);
double  or_rmsd_lower(or_ctx*, int lig, const double* xyz_a, const double* xyz_b);

/* Optimisers (conf in/out), return final energy; *evals counts f(x) calls. */
double  or_rilc_bfgs(or_ctx*, int lig, double* conf, const double v[3], double slope,
                     int max_steps, int64_t* evals);
double  or_bfgs(or_ctx*, int lig, double* conf, const double v[3], double slope,
                int max_steps, int use_noncache, int64_t* evals);

typedef struct {
    uint32_t seed;
    uint32_t lig_uid;        /* RNG stream id of the ligand                 */
    int32_t  search_depth;   /* MC steps per chain                          */
    int32_t  max_bfgs_steps;
    double   hunt_cap[3];    /* (10,10,10) as main.cpp:395                  */
    double   slope;          /* 1e6                                         */
    double   temperature;    /* 1.2                                         */
    double   amplitude;      /* 2                                           */
    int32_t  dense;          /* 0: RILC-BFGS local search (--rilc_bfgs 1);
                                1: dense BFGS (--rilc_bfgs 0)               */
    int32_t  visited;        /* 1: QuickVina2-CUDA's visited history (RILC
                                only): a chain runs its first 10*(6+ntors)
                                local optimisations, later candidates keep
                                their entry energy (visited.cuh:48-227,
                                quasi_newton.cuh:1937-1943)                  */
} or_search;

/* Runs chains [chain_begin, chain_end) of the Monte-Carlo search
 * (kernel2.cu:219-426 semantics for RILC-BFGS, 427-563 for dense BFGS;
 * Philox streams shared with the GPU code).
 * out_conf: [n*(7+ntors)], out_e: [n]; threads: host threads to use. */
int64_t or_mc_chains(or_ctx*, int lig, const or_search*, int chain_begin, int chain_end,
                     double* out_conf, double* out_e, int threads);
void    or_init_conf(or_ctx*, int lig, uint32_t seed, uint32_t lig_uid, uint32_t chain,
                     double* conf);
/* Refinement as main.cpp:139-157 (slope ramp, dense BFGS on the direct sum). */
double  or_refine(or_ctx*, int lig, double* conf, int max_steps, int64_t* evals);

/* Greedy diversity clustering over energy-sorted results: keeps up to
 * max_keep poses whose heavy-atom RMSD to every kept pose is >= min_rmsd. */
int     or_cluster(or_ctx*, int lig, int n, const double* confs, const double* e,
                   double min_rmsd, int max_keep, int32_t* kept_idx);

/* Cell-list grid builder timing helper (cache.cpp:148-208 over all points). */
double  or_grid_seconds(or_ctx*, const int32_t* types, int n_types, int threads);

/* Philox4x32-10 (Salmon et al. 2011), exposed so tests can pin the stream. */
void    or_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

#ifdef __cplusplus
}
#endif
#endif
