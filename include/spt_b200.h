/*
 * spt_b200.h -- C ABI of the B200 (sm_100a) backend for the
 * specific_particle_tracer hot path (AdamCBartnik/BEM).
 *
 * Plain C: fixed-width integers, doubles and raw pointers only.  Every data
 * pointer is a DEVICE pointer on the current CUDA device unless a comment
 * says otherwise; the caller allocates and owns all of them (the library
 * never frees caller memory).  Every entry point returns SPT_OK (0) or an
 * error code, and records a message readable with spt_last_error().  A
 * call enqueues work on `stream` (a cudaStream_t passed as void*; NULL is
 * the legacy default stream) and does not synchronise.
 *
 * Reference interfaces each entry point replaces (paths inside the
 * reference project):
 *   spt_trace      batched_rk45.integrate(accel_fn, pos0, vel0, t_birth, t_max,
 *                  rtol, atol, kill_fn=...)            batched_rk45.py:55-323
 *                  with accel_fn = geometry.make_accel_fn(...) geometry.py:265-301
 *                  and kill_fn = geometry.make_kill_fn(...) geometry.py:304-322
 *   spt_accel      the accel(pos, vel, active, group_idx) closure geometry.py:289-299
 *   spt_bem_field  AxisymmetricBEMSolution.field(points)  bem/axisymmetric.py:474-487
 *                  -> evaluate_axisymmetric_field         bem/axisymmetric.py:501-605
 *   spt_surrogate_field  the learned-form field (no reference counterpart:
 *                  an MLP stand-in for evaluate_axisymmetric_field, exact
 *                  within a band around the surface)
 *   spt_ring_field ring_field(rho, z, a)                  bem/axisymmetric.py:235-265
 *   spt_ellip_ke   ellip_ke_complement(p)                 bem/_elliptic.py:28-39
 *   spt_bem_assemble  the collocation matrix of AxisymmetricBEMSolution.solve
 *                  (adaptive _segment_potential)          bem/axisymmetric.py:275-302, 411-443
 */
#ifndef SPT_B200_H
#define SPT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPT_ABI_VERSION 4

/* return codes */
#define SPT_OK 0
#define SPT_ERR_ARG 1        /* invalid argument (shape, size, null pointer, alignment) */
#define SPT_ERR_CUDA 2       /* a CUDA runtime call failed */
#define SPT_ERR_CAPACITY 3   /* a size exceeds a documented maximum */

/* geometry kinds (Geometry subclasses of geometry.py / bem/geometry.py) */
#define SPT_GEOM_FLAT 0      /* geometry.FlatCathode                       geometry.py:97-163 */
#define SPT_GEOM_TIP 1       /* geometry.HemisphericalTip                  geometry.py:166-256 */
#define SPT_GEOM_TIP_BEM 2   /* bem.geometry.HemisphericalTipBEMGeometry, z0=None  bem/geometry.py:58-507 */
#define SPT_GEOM_WELL_BEM 3  /* bem.geometry.CylindricalWellBEMGeometry, z0=None   bem/geometry.py:510-885 */
#define SPT_GEOM_POST_BEM 4  /* hemisphere on a cylindrical post: capsule BEM field, 3-image force in the apex frame */

/* arithmetic forms */
#define SPT_FORM_FP64 0      /* plain: float64 throughout */
#define SPT_FORM_MIXED 1     /* pair and BEM panel sums in float32 with Kahan compensation */
#define SPT_FORM_SURROGATE 2 /* mixed, with the BEM field of points outside a near-surface band
                                taken from the learned MLP surrogate (tensor cores) */

/* per-group status (SptState.status) */
#define SPT_GROUP_NEW 0      /* not started: t, h are initialised on first touch */
#define SPT_GROUP_RUNNING 1
#define SPT_GROUP_DONE 2     /* t >= t_max (1 - 1e-14)  (batched_rk45.py:317) */
#define SPT_GROUP_NONFINITE 3/* the error norm became NaN: group stopped */
#define SPT_GROUP_TIMEOUT 4  /* a bounded device wait gave up (TMA tile never arrived) */

/* SptTraceParams.team */
#define SPT_TEAM_AUTO 0
#define SPT_TEAM_CTA 1
#define SPT_TEAM_WARP 2

/* device counters (SptTraceParams.counters, accumulated, uint64) */
#define SPT_CNT_ATTEMPTS 0           /* group-step attempts */
#define SPT_CNT_ACCEPTED 1           /* accepted group-steps */
#define SPT_CNT_PARTICLE_STEPS 2     /* sum over accepted group-steps of the group size */
#define SPT_CNT_STAGE_EVALS 3        /* particle-stage evaluations (7 per particle-attempt) */
#define SPT_CNT_PAIR_EVALS 4         /* pair interactions summed (all image sets included) */
#define SPT_CNT_RING_FAR 5           /* far-quadrature ring-kernel evaluations */
#define SPT_CNT_RING_NEAR 6          /* near (sinh-quadrature) ring-kernel evaluations */
#define SPT_CNT_NEAR_PAIRS 7         /* (point, segment) pairs handled by the near quadrature */
#define SPT_CNT_FP64_ROUNDS 8        /* mixed form: far-sum rounds recomputed in float64 (ill-conditioned) */
#define SPT_CNT_FP64_TARGETS 9       /* mixed form: pair-sum targets recomputed in float64 */
#define SPT_CNT_LIVE_STEPS 10        /* sum over accepted group-steps of the particles alive (born, not
                                        killed) at the step start */
#define SPT_CNT_CLUSTER_EVALS 11     /* cluster-expansion evaluations of the adaptive far rule */
#define SPT_N_COUNTERS 12

/* Geometry parameters.  Fields a kind does not use are ignored. */
typedef struct {
    int32_t kind;            /* SPT_GEOM_* */
    int32_t has_image;       /* image-charge force on (z0 given) */
    int32_t has_kill_below;  /* kill at z <= kill_z_below */
    int32_t has_z_max;       /* kill at z >= z_max (geometry.make_kill_fn) */
    double E_gun;            /* asymptotic field Ez [V/m] */
    double R;                /* tip / post / well radius [m] */
    double H;                /* well depth [m] */
    double L;                /* post height = apex sphere centre z [m] */
    double z0;               /* image-plane recession [m] */
    double kill_z_below;
    double z_max;
    double z_handoff;        /* BEM below z_handoff/2, flat fallback above z_handoff */
    double bottom_fillet;    /* well corner rounding radii [m] (0 = sharp) */
    double rim_fillet;
} SptGeometry;

/* Number of per-segment fields in SptBem.seg (structure of arrays, each
 * n_seg doubles, row stride seg_stride):
 *   0 p0_rho  1 p0_z  2 tan_rho  3 tan_z   (tan = p1 - p0)
 *   4 length  5 unit_rho  6 unit_z  7 normal_rho  8 normal_z
 *   9 sigma0 (density at p0)  10 sigma1 (density at p1)              */
#define SPT_SEG_FIELDS 11

/* Largest azimuthal mode n_max the image-charge entry points accept. */
#define SPT_IMAGE_MAX_MODES 64

/* Tables of one image-charge solution (ImageChargeBEMSolution,
 * bem/image_charge.py:457-620), built once per geometry by the host. */
typedef struct {
    int32_t n_nodes;          /* P profile nodes (at least 2) */
    int32_t n_max;            /* modes 0..n_max, at most SPT_IMAGE_MAX_MODES */
    int32_t n_quad;           /* reconstruction nodes: (P-1) * n_subdiv * 4 */
    int32_t mirror_symmetric; /* profile mirror-doubled through z = -z0 (image_mirror_symmetric=True):
                                 phantom sources (z -> -2 z0 - z, -q) join the solve, the plane image is
                                 added back, and a source whose plane is nearer than the profile takes
                                 no local mirror charge (bem/geometry.py:346-415, image_charge.py:538-585) */
    const double* node;       /* [2][P]: rho (floored at rho_floor), z of the profile nodes */
    const double* seg;        /* [6][P-1]: p0_rho p0_z tan_rho tan_z normal_rho normal_z (tan = p1 - p0) */
    const double* quad;       /* [5][n_quad]: rho z length-weight t segment-index (image_charge.py:418-452) */
    const double* a_inv;      /* [(n_max+1) x P x P] row-major: the inverse of each mode's operator */
    double rho_floor;         /* 1e-6 * max profile rho */
    double d_lo, d_hi;        /* mirror-charge blend distances [m] (image_charge_weight; d_hi <= d_lo: no mirror) */
} SptImage;

/* Precomputed BEM solution tables (bem/axisymmetric.py:305-338, 490-498).
 * `node` holds 3 rows of node_stride doubles: rho_q, z_q, w_q = area_q*sigma_q
 * for the n_seg*nodes_per_seg Gauss-4 far-quadrature nodes, segment-major.
 * node_stride must be even (16-byte rows); the device pointers must be
 * 16-byte aligned (tiles are copied with the TMA bulk engine). */
typedef struct {
    int32_t n_seg;
    int32_t nodes_per_seg;   /* 4 * n_subdiv, at most 256 */
    int64_t seg_stride;
    int64_t node_stride;
    const double* seg;
    const double* node;
    double gauss8_x[8];      /* Gauss-Legendre 8-point nodes/weights on [-1, 1] */
    double gauss8_w[8];
    /* Far-field rule (no counterpart in the reference, which always uses the
     * first): SPT_FAR_REFERENCE sums every far segment over its
     * nodes_per_seg nodes; SPT_FAR_ADAPTIVE classifies each segment, per
     * round of up to 8 evaluation points, by the smallest distance / length
     * ratio over the round: below ratio4 the reference nodes, below ratio2
     * the 4-point Gauss rule over the whole segment, else the 2-point rule.
     * `coarse` holds 3 rows (rho_q, z_q, w_q) of coarse_stride doubles with
     * 6 nodes per segment: the 4 Gauss-4 nodes, then the 2 Gauss-2 nodes.
     * ratio4 >= 1 (coarse segments are never near), ratio2 >= ratio4. */
    int32_t far_rule;
    int32_t reserved;
    double ratio4;
    double ratio2;
    const double* coarse;
    int64_t coarse_stride;
    /* Optional bounds of each run of SPT_BLOCK_SEGS consecutive segments,
     * 6 rows of blk_stride doubles: centre rho, centre z, radius (largest
     * distance from the centre to an endpoint of the run), largest segment
     * length, arclength of the run, and 1 where the run may take the run
     * rule below (else 0).  With it the closest-segment search, the near
     * test and the adaptive classification skip runs that cannot qualify
     * (results are unchanged); NULL scans every segment. */
    const double* blk;
    int64_t blk_stride;
    /* Run rule (adaptive far rule with blk only): a run flagged in blk row 5
     * whose lower-bound distance over the round is at least ratio_run times
     * its arclength takes the 8-point Gauss rule over the whole run.
     * run_nodes holds 3 rows (rho_q, z_q, w_q) of run_stride doubles, 8 nodes
     * per run.  ratio_run <= 0 turns the rule off. */
    double ratio_run;
    const double* run_nodes;
    int64_t run_stride;
    /* Cluster expansions (adaptive far rule with blk only; no counterpart in
     * the reference): a binary tree over the runs -- level 0 the runs, level
     * l the clusters of 2^l consecutive runs, ceil(n_run / 2^l) of them,
     * levels stored one after another -- with, per cluster, a record of
     * cluster_terms + 2 doubles: the centre z_c on the axis, the radius
     * r_max of the sphere about (0, z_c) that holds all its rings, and the
     * axisymmetric multipole moments M_n = sum_q w_q (r_q / r_max)^n
     * P_n(cos theta_q) of its reference nodes (n < cluster_terms).  A run
     * whose cluster at some level is at least cluster_kappa * r_max from the
     * point is summed by the highest such cluster's expansion
     * E = -grad (1/4 pi) sum_n M_n r_max^n P_n(cos theta) / r^(n+1), which
     * matches the reference nodes' sum to ~1e-15 of the cluster's field at
     * kappa 3, 32 terms.  cluster_kappa <= 0 or clusters NULL: off.
     * At most SPT_MAX_CLUSTER_RUNS runs, 64 terms. */
    const double* clusters;
    int32_t cluster_levels;
    int32_t cluster_terms;
    double cluster_kappa;
    /* BEM image-charge force (geometries built with z0: kind SPT_GEOM_TIP_BEM
     * or SPT_GEOM_WELL_BEM with has_image): the tables of the image profile's
     * mode solve.  spt_trace and spt_accel add the geometry-level force of
     * spt_image_force to every stage (n_max at most SPT_TRACE_IMAGE_MODES
     * there); n_nodes = 0: none. */
    SptImage image;
} SptBem;

/* Largest image-charge n_max inside spt_trace / spt_accel. */
#define SPT_TRACE_IMAGE_MODES 16

#define SPT_MAX_CLUSTER_RUNS 256

#define SPT_RUN_NODES 8

#define SPT_BLOCK_SEGS 32

#define SPT_FAR_REFERENCE 0
#define SPT_FAR_ADAPTIVE 1

/* Particle and per-group integrator state, in/out. Groups are contiguous
 * particle ranges [group_offset[g], group_offset[g+1]). */
typedef struct {
    int32_t n_groups;
    int32_t max_group_size;  /* max over g of group size */
    int64_t n_particles;
    const int64_t* group_offset;   /* [n_groups+1] */
    const int32_t* group_order;    /* [n_groups] processing order (e.g. largest first) or NULL */
    double* x; double* y; double* z;
    double* vx; double* vy; double* vz;
    const double* t_birth;
    double* t_death;               /* +inf while alive; set to the step end time when killed */
    const double* charge;          /* signed charge [C] */
    const double* mass;            /* per-particle mass [kg] */
    double* t;                     /* [n_groups] group clock */
    double* h;                     /* [n_groups] next step size */
    int32_t* status;               /* [n_groups] SPT_GROUP_* */
    int64_t* n_accepted;           /* [n_groups] */
    int64_t* n_rejected;           /* [n_groups] */
    /* Optional device count: process only group_order[0, *n_active) (the
     * running groups after spt_compact_groups; lets a captured CUDA graph
     * shrink its work without host involvement).  NULL: all n_groups.
     * Needs group_order. */
    const int32_t* n_active;
} SptState;

typedef struct {
    double t_max, rtol, atol;
    double plummer_radius;
    double charge_to_mass;         /* species q/m for the external-field term */
    double coulomb_constant;       /* 1/(4 pi eps0) [N m^2 C^-2] (constants.py:14) */
    double safety, min_factor, max_factor, initial_step_fraction;
    int64_t max_attempts;          /* attempts per group in this call */
    int32_t form;                  /* SPT_FORM_* */
    int32_t log_capacity;          /* entries per group in log_h/log_err (0: no log) */
    double* log_h;                 /* [n_groups][log_capacity] step used by attempt k */
    double* log_err;               /* [n_groups][log_capacity] its error norm */
    unsigned long long* counters;  /* [SPT_N_COUNTERS] or NULL */
    /* screens (screens.py:43-168): z planes; every crossing inside an accepted
     * step is located on the step's cubic Hermite z(s) (split at its extrema,
     * 60 bisection steps) and appended to screen_rec, a [9][screen_capacity]
     * array of (t, x, y, z, vx, vy, vz, screen index, particle index);
     * screen_count counts every crossing found, including any beyond the
     * capacity (which are dropped). */
    int32_t n_screens;
    int32_t n_outputs;
    const double* screens;
    double* screen_rec;
    int64_t screen_capacity;
    unsigned long long* screen_count;
    /* output times (batched_rk45.py:186-209, 295-312; trajectories.py:44-74):
     * ascending; every group's step lands on each one exactly; the state of
     * every particle born by then is written to output_rec
     * [n_outputs][7][n_particles] (t, x, y, z, vx, vy, vz) and flagged in
     * output_flag [n_outputs][n_particles]. */
    const double* output_times;
    double* output_rec;
    uint8_t* output_flag;
    /* learned form (SPT_FORM_SURROGATE, BEM geometries): MLP with inputs
     * (log distance d to the profile, arclength position of the closest
     * profile point) and outputs (E_normal, E_tangent) / (|sigma| + floor) /
     * g(d).  sur_w: FP32 (BF16-rounded) parameters W1[128x2] b1 W2[128x128]
     * b2 W3 b3 W4 b4 W5[2x128] b5, flat; sur_w16: the same in BF16 (the
     * tensor-core layers read W2..W4 from it); sur_s_start[n_seg]: arclength
     * at each segment start; sur_log_scale[64]: ln g on a uniform grid of
     * ln d over [sur_d_min, sur_d_max].  Points closer than sur_band to the
     * profile use the exact BEM sum, and so does a hashed sur_spot fraction
     * of the others, whose surrogate error is recorded in sur_stats
     * [surrogate points, exact points, spot checks, max relative error
     * (float bits)]. */
    const float* sur_w;
    const void* sur_w16;
    const double* sur_s_start;
    const double* sur_log_scale;
    double sur_s_end, sur_sig_floor, sur_band, sur_spot, sur_d_min, sur_d_max;
    unsigned long long* sur_stats;
    /* Far-sum tile shape of the reference far rule: evaluation points per
     * round, 1, 2 or 4 (0 or anything else: 4).  Fewer points per round give
     * each thread more nodes in flight per point; more points share each
     * node load.  Results agree to rounding.  (The adaptive rule takes one
     * point per warp task, classified for that point alone.) */
    int32_t round_points;
    /* CTA width of the trace: 32, 64, 128 or 256 threads work on one group
     * at a time (0 or anything else: by group size -- 64 up to 16
     * particles, 128 up to 64, else 256; 256 with the reference far rule;
     * at least 128 for the learned form).  Narrower CTAs put more groups on
     * an SM and fewer warps behind each barrier.  Results do not depend on
     * it beyond the summation order of the reductions. */
    int32_t cta_threads;
    /* Mixed form: a float32 far-sum round or pair sum whose sum of |terms|
     * exceeds kappa_max times the whole field (uniform included) or the
     * whole acceleration at a point is recomputed in float64 -- the float32
     * result would carry eps_f x that ratio of relative error (shielded
     * regions, where the perturbation cancels the uniform field; dense
     * bunches).  0: the default, 16. */
    double kappa_max;
    /* Largest persistent grid (CTAs) of this launch; 0: the whole GPU (SMs x
     * resident CTAs).  Launches of different group-size bins on concurrent
     * streams share the SMs by giving each a grid in proportion to its work. */
    int32_t max_ctas;
    /* Team that advances one group: SPT_TEAM_AUTO (0) lets the library
     * choose; SPT_TEAM_CTA (1) keeps one group per CTA; SPT_TEAM_WARP (2)
     * asks for one group per warp (lane i = particle i, several groups per
     * CTA, no CTA barrier inside a group's step), offered for BEM geometries
     * without the BEM image-charge force, groups of at most 32 particles,
     * the float64 form and the adaptive far rule -- the case AUTO gives to
     * the warp team whenever the workspace holds its slope slots. */
    int32_t team;
} SptTraceParams;

/* Scratch bytes spt_trace needs for this state/geometry (work-queue
 * counter, and per-CTA group buffers when a group does not fit shared
 * memory). Host-only; no device work. */
int spt_trace_workspace_bytes(const SptState* state, const SptTraceParams* params,
                              const SptGeometry* geom, const SptBem* bem, int64_t* bytes);

/* Advance every group with status NEW or RUNNING by at most
 * params->max_attempts Dormand-Prince 5(4) attempts (one persistent kernel,
 * one CTA per group at a time, groups taken from a device work queue).
 * `bem` may be NULL for SPT_GEOM_FLAT / SPT_GEOM_TIP. `workspace` is a
 * device buffer of at least spt_trace_workspace_bytes() bytes, 256-byte
 * aligned; the call clears what it needs. */
int spt_trace(const SptState* state, const SptTraceParams* params, const SptGeometry* geom,
              const SptBem* bem, void* workspace, int64_t workspace_bytes, void* stream);

/* One stage evaluation (the accel closure): acc = (q/m)_s E(pos)
 * + F_coulomb/m + F_image/m on active particles, 0 elsewhere.
 * pos_*, acc_* are [n_particles]; active is uint8 [n_particles]. */
typedef struct {
    int32_t n_groups;
    int32_t max_group_size;
    int64_t n_particles;
    const int64_t* group_offset;
    const double* x; const double* y; const double* z;
    const uint8_t* active;
    const double* charge;
    const double* mass;
    double charge_to_mass;
    double coulomb_constant;
    double plummer_radius;
    int32_t form;
    double* ax; double* ay; double* az;
} SptAccelArgs;
int spt_accel(const SptAccelArgs* args, const SptGeometry* geom, const SptBem* bem, void* stream);

/* Compaction of retired groups: out[0, *n_active) = the entries g of
 * order[0, n) (the identity when order is NULL) with status[g] <
 * SPT_GROUP_DONE, in order.  out may alias order.  One CTA; no host sync,
 * so it can be captured in a CUDA graph with the spt_trace calls that
 * follow it. */
int spt_compact_groups(const int32_t* order, int32_t n, const int32_t* status, int32_t* out, int32_t* n_active,
                       void* stream);

/* Perturbation field E = -grad S[sigma] of the BEM solution at n points
 * (x, y, z) -> (ex, ey, ez), all [n] device arrays. */
int spt_bem_field(const double* x, const double* y, const double* z, int64_t n, const SptBem* bem,
                  int32_t form, double* ex, double* ey, double* ez, void* stream);

/* Learned-form perturbation field at n points: the surrogate MLP (sur_*
 * fields of `sur`; the other fields are ignored) outside sur_band metres of
 * the profile, the exact sum of spt_bem_field (mixed form) inside it and for
 * the sur_spot fraction of points spot-checked, statistics into sur_stats
 * when it is not NULL.  Same device code as the learned-form stages of
 * spt_trace. */
int spt_surrogate_field(const double* x, const double* y, const double* z, int64_t n, const SptBem* bem,
                        const SptTraceParams* sur, double* ex, double* ey, double* ez, void* stream);

/* Unit-charge ring field (E_rho, E_z) at (rho, z) for ring radius a; [n]. */
int spt_ring_field(const double* rho, const double* z, const double* a, int64_t n, int32_t form,
                   double* er, double* ez, void* stream);

/* K(1-p), E(1-p) for p in (0, 1]; [n]. */
int spt_ellip_ke(const double* p, int64_t n, int32_t form, double* K, double* E, void* stream);

/* Collocation matrix of the P1 single-layer BEM on a generating profile
 * (bem/axisymmetric.py:411-443): A [n_nodes x n_nodes], row-major, A[i][j] =
 * potential at node i of the unit hat density of node j, by adaptive
 * bisection (refine while segment length > refine_ratio * distance, up to
 * max_depth levels) with the 4-point Gauss rule (gauss4_x/w, device arrays of
 * 4) on each leaf.  profile_rho/z are [n_nodes] device arrays. */
int spt_bem_assemble(const double* profile_rho, const double* profile_z, int32_t n_nodes, double refine_ratio,
                     int32_t max_depth, const double* gauss4_x, const double* gauss4_w, double* A, void* stream);

/* ---- BEM image-charge force (azimuthal Fourier modes) ------------------
 * The induced-charge force of an axisymmetric grounded conductor on the
 * particles of each group (bem/image_charge.py, bem/ring_modes.py,
 * bem/toroidal.py; used by bem/geometry.py:326-344, 780-797 when a BEM
 * geometry is built with z0). */


/* Toroidal harmonics Q_{m-1/2}(chi) and dQ_{m-1/2}/dchi, m = 0..n_max, for
 * chi >= 1 (clipped to the next double above 1): q, dq are [(n_max+1) x n]
 * row-major.  Replaces toroidal_Q, bem/toroidal.py:180-219. */
int spt_toroidal_q(const double* chi, int64_t n, int32_t n_max, double* q, double* dq, void* stream);

/* Per-mode single-layer collocation operators of a generating profile:
 * A [(n_max+1) x n_nodes x n_nodes] row-major, A[m][i][j] = mode-m
 * potential at node i (rho floored at rho_floor, which the reference sets
 * to 1e-6 max rho) of the unit hat density
 * of node j, by the adaptive bisection of spt_bem_assemble with the mode
 * kernel Phi_m on each Gauss-4 leaf.  Replaces assemble_mode_operators,
 * bem/image_charge.py:379-411, 470-495. */
int spt_image_assemble(const double* profile_rho, const double* profile_z, int32_t n_nodes, int32_t n_max,
                       double rho_floor, double refine_ratio, int32_t max_depth, const double* gauss4_x,
                       const double* gauss4_w, double* A, void* stream);


/* Image-charge force on the particles of every group, [n_particles]:
 * the joint per-group solve of ImageChargeBEMSolution.image_force
 * (bem/image_charge.py:816-1056) -- local mirror charges, per-mode RHS,
 * sigma = A^-1 rhs, field on the fixed quadrature, direct mirror field.
 * With geom == NULL that solution-level force alone (in N); with a geometry
 * (kind SPT_GEOM_TIP_BEM or SPT_GEOM_WELL_BEM, has_image set) the
 * geometry's image_force: the flat plane image at geom->z0 above
 * geom->z_handoff, the BEM image force below z_handoff / 2, smoothstep
 * between (plummer_radius softens the plane image).  Inactive particles
 * (active[i] == 0) neither excite the solve nor feel a force.  At most 512
 * particles per group (256 with mirror_symmetric).  Shared memory per CTA:
 * 8 * (10 S + 3 E + 2 (1 + c) (n_max+1) n_nodes) bytes, S = E (2E with
 * mirror_symmetric) sources, c in [1, 8] partial right-hand sides; it must
 * fit 227 KB with c = 1 (SPT_ERR_CAPACITY otherwise). */
int spt_image_force(const double* x, const double* y, const double* z, const double* charge, const uint8_t* active,
                    const int64_t* group_offset, int32_t n_groups, int32_t max_group_size, const SptImage* image,
                    const SptGeometry* geom, double coulomb_constant, double plummer_radius, double* fx, double* fy,
                    double* fz, void* stream);

/* spt_trace for callers that cannot allocate device memory: a caller with no
 * device allocator of its own (a cgo/JNI/ctypes binding without torch), or
 * one running where a cudaMalloc would implicitly synchronise the device and
 * stall other streams, or one whose device memory is fully reserved by
 * another framework's pool.  Same state, parameters and results as
 * spt_trace, but no workspace: the scratch is a fixed 4 MiB device array
 * inside the library, held on every GPU that loads the library until the
 * process exits.  No counterpart in the reference.
 *   - max_group_size must be in [1, 1024] (SPT_ERR_CAPACITY otherwise); for
 *     groups above 256 particles the scratch holds floor((4 MiB - 256) /
 *     (432 * max_group_size)) per-CTA buffers, which caps the number of
 *     CTAs that run at once (9 at 1024 particles).
 *   - The warp team (SptTraceParams.team) keeps 13,824 bytes per warp of
 *     step state in the same scratch, which holds 37 CTAs of 256 threads:
 *     SPT_TEAM_AUTO keeps one group per CTA here (the warp team takes only
 *     launches that fill the GPU, whose grid does not fit), and an explicit
 *     SPT_TEAM_WARP runs on those 37 CTAs.
 *   - The first call in each CUDA context (the current device's primary
 *     context, or the caller's own driver-API context) looks the array's
 *     address up (cudaGetSymbolAddress) with that device current and caches
 *     it under the context's id; make that first call before any stream
 *     capture.  After a device reset the next call looks it up again.
 *   - Every call shares the one array: calls that overlap on the GPU (other
 *     streams, other host threads) race on it; serialise them.  Each call
 *     clears the work-queue counter it needs; nothing else carries over. */
int spt_trace_noalloc(const SptState* state, const SptTraceParams* params, const SptGeometry* geom,
                      const SptBem* bem, void* stream);

/* ---- learned field surrogate: BF16 tensor-core MLP kernels (no counterpart
 * in the reference; they train and evaluate the (rho, z) -> (E_rho, E_z)
 * surrogate of the BEM field).  Return 0, 1 (bad argument) or 2 (launch). */
#define SPT_EPI_STORE 0       /* C = acc (FP32), per K split at C + split * split_stride */
#define SPT_EPI_BIAS_SILU 1   /* C = z = acc + bias (FP32, optional), H = SiLU(z) (BF16) */
#define SPT_EPI_DSILU 2       /* H = acc * SiLU'(Z) (BF16) */
typedef struct {
    int32_t M, N, K;          /* D[M x N] = A[M x K] B[N x K]^T; K a multiple of 64 (of 64 * split_k) */
    int32_t a_mn, b_mn;       /* 0: element (r, k) at X[r*ld + k]; 1: at X[k*ld + r] */
    int32_t epi, split_k, reserved;
    int64_t lda, ldb, ldc, split_stride;   /* lda, ldb multiples of 8 */
    const void* A;            /* BF16, 16-byte aligned */
    const void* B;            /* BF16, 16-byte aligned */
    float* C;
    const float* bias;
    const float* Z;
    void* H;                  /* BF16 */
    int32_t* status;          /* set to 1 if a bounded wait gave up (optional) */
} SptGemmArgs;
int spt_mlp_gemm(const SptGemmArgs* args, void* stream);
int spt_mlp_first_layer(const float* x, int64_t n, const float* W1, const float* b1, float* z, void* h, void* stream);
int spt_mlp_last_layer(const void* h, const float* z, int64_t n, const float* W5, const float* b5, float* y,
                       const float* target, float inv_batch, void* delta, float* dW5, float* db5, float* loss,
                       void* stream);
int spt_mlp_colsum(const void* delta, int64_t n, const float* x, float* db, float* dW1, void* stream);
int spt_mlp_reduce_splits(const float* part, int32_t splits, int64_t n, float* out, void* stream);
int spt_mlp_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float beta1, float beta2,
                 float eps, int32_t step, void* p_bf16, float* p_rounded, void* stream);

/* Last error message of the calling thread (NUL-terminated, truncated to
 * len). Returns the length of the full message. */
int spt_last_error(char* buf, int32_t len);

/* SPT_ABI_VERSION. */
int spt_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* SPT_B200_H */
