/*
 * titan_b200.h — C ABI of the B200 (sm_100a) plasma time step of TITAN.
 *
 * Drop-in replacement for the two OpenMP loops of
 *   void Setka::Go(bool is_inner_area, size_t steps, short metod)
 *        (TITAN/source/Setka.h:221, body TITAN/source/Setka_physics.cpp:1484-2278)
 * i.e. the per-face flux loop
 *   double Setka::Culc_Gran_Potok(Gran*, unsigned short now, short metod, string&, const double& time)
 *        (TITAN/source/Setka.h:223, TITAN/source/Setka_physics.cpp:2280-2571)
 * with its reconstruction Setka::Snos_on_Gran (TITAN/source/Setka_gran_snos.cpp:3-1075)
 * and Riemann solver Phys_param::chlld (TITAN/source/Phys_param.h:240-251,
 * TITAN/source/Phys_param.cpp:882-1878), the per-cell conservative update with
 * the charge-exchange sources Setka::Calc_sourse_MF_Bera
 * (TITAN/source/Setka_physics.cpp:766-1258), the CFL reduction and the
 * geometry refresh Setka::Calculating_measure (TITAN/source/Setka.cpp:2465-2502).
 *
 * Conventions (all arrays are host memory owned by the caller and copied at
 * the call; nothing is retained after a call returns):
 *   - indices are 0-based (the reference's `number` minus 1);
 *   - cell state is SoA [TITAN_NV][ncell]: rho, Vx, Vy, Vz, p, Bx, By, Bz, Q,
 *     rho_He — the names of Cell::parameters (TITAN/source/Cell.h:36), B in
 *     Gaussian units as the reference stores it;
 *   - every call returns a titan_status; on failure titan_last_error() gives a
 *     message. The library never exits the process (the reference's
 *     convention is print + exit(-1)).
 * One host thread per context; calls on a context are synchronous.
 */
#ifndef TITAN_B200_H
#define TITAN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TITAN_NV 10

typedef enum titan_status {
    TITAN_OK = 0,
    TITAN_EINVAL = -1,      /* bad argument */
    TITAN_EMESH = -2,       /* mesh fails a consistency check (Setka::Test_geometr rules) */
    TITAN_ENONFINITE = -3,  /* NaN / subnormal produced (the reference's Error 9851234578) */
    TITAN_ECUDA = -4,       /* CUDA runtime error */
    TITAN_ETIMEOUT = -5,    /* a bounded device wait gave up */
    TITAN_ENOMEM = -6,      /* device allocation failed */
    TITAN_ESOLVER = -7      /* Riemann solver found no admissible wave region */
} titan_status;

/* Type_Gran (TITAN/source/Gran.h:5-10) */
enum { TITAN_FACE_US = 0, TITAN_FACE_INNER_HARD = 1, TITAN_FACE_OUTER_HARD = 2, TITAN_FACE_OUTER_SOFT = 3 };
/* Type_Gran_surf (TITAN/source/Gran.h:12-17) */
enum { TITAN_SURF_US = 0, TITAN_SURF_TS = 1, TITAN_SURF_HP = 2, TITAN_SURF_BS = 3 };
/* Type_Cell (TITAN/source/Cell.h:5-11) */
enum { TITAN_CELL_NONE = 0, TITAN_CELL_ZONE_1 = 1, TITAN_CELL_ZONE_2 = 2, TITAN_CELL_ZONE_3 = 3, TITAN_CELL_ZONE_4 = 4 };
/* n_state of Phys_param::chlld */
enum { TITAN_LAX = 0, TITAN_HLL = 1, TITAN_HLLC = 2, TITAN_HLLD = 3 };

/* Flattened Setka: All_Yzel / All_Cell / All_Gran (TITAN/source/Setka.h:8-322). */
typedef struct titan_mesh {
    int64_t nnode, ncell, nface, nbc;
    const double*  node_xyz;    /* [nnode*3]  Yzel::coord[0] */
    const int32_t* cell_nodes;  /* [ncell*8]  Cell::yzels */
    const int32_t* cell_faces;  /* [ncell*6]  Cell::grans, order kept (flux gather order) */
    const int8_t*  cell_type;   /* [ncell]    Cell::type */
    const uint8_t* cell_tvd;    /* [ncell]    Cell::is_TVD (B frozen where 0) */
    const int32_t* face_nodes;  /* [nface*4]  Gran::yzels, around the quad */
    const int32_t* face_cells;  /* [nface*2]  Gran::cells; -1 when the face has one cell */
    const int8_t*  face_type;   /* [nface]    Gran::type */
    const int8_t*  face_surf;   /* [nface]    Gran::type2 */
    const int32_t* face_bc;     /* [nface]    row of bc_vals for hard boundary faces, else -1 */
    const double*  bc_vals;     /* [nbc*TITAN_NV] fixed face values (Gran::parameters) */
    const double*  node_amp;    /* [nnode] or NULL: prescribed radial node speed amplitude */
    const double*  node_phase;  /* [nnode] or NULL: its phase */
} titan_mesh;

/* Phys_param settings that the step reads (TITAN/source/Phys_param.h:95-160). */
typedef struct titan_params {
    double gamma;          /* adiabatic index (5/3) */
    double KFL;            /* Courant number */
    double velosity_inf;   /* Velosity_inf, used by the Outer_Soft outflow fix-up */
    double omega;          /* angular frequency of the prescribed node motion */
    double par_a_2;        /* charge-exchange cross-section parameter */
    double par_n_H_LISM;   /* n_H at infinity */
    double par_Kn;         /* Knudsen number */
    double beta_switch;    /* method_policy 1: HLLD where B^2/(8 pi p) > beta_switch, else HLLC */
    int32_t move;          /* move_setka: ALE step with prescribed node motion */
    int32_t soft_fixups;   /* Outer_Soft outflow fix-ups (1, as the reference) or plain copy (0) */
    int32_t method_policy; /* 0: per-face n_state from titan_set_face_method; 1: beta switch */
    int32_t npassive;      /* 0, or 2 to carry Q and rho_He through the contact */
    int32_t nh;            /* frozen neutral fluids for the Bera sources (0..4) */
    int32_t TS_hard;       /* left_ydar on TS faces */
    int32_t contact_hard;  /* face speed = contact speed on HP faces */
    int32_t flux_precision;/* 64: all-FP64; 32: FP32 Riemann-solver arithmetic (faces wholly in one
                              side's wave region take that side's FP64 flux), FP64 flux records,
                              accumulation, update, pressure recovery and dt */
    int32_t tvd;           /* Phys_param::TVD: second-order reconstruction on interior faces
                              (Setka_gran_snos.cpp:188-735; neighbours from Setka::Init_TVD) */
    int32_t snos_on_hp;    /* Phys_param::Snos_on_HP: second order on HP faces too */
    int32_t bn_in_p_on_hp; /* Phys_param::bn_in_p_on_HP: on HP faces the magnetic pressure goes into p
                              and the exact gas-dynamic solver Godunov_Solver_Alexashov runs
                              (Setka_physics.cpp:2378-2409, Phys_param.cpp:1938-2385) */
} titan_params;

typedef struct titan_step_info {
    int64_t steps_done;      /* steps completed by this call */
    int64_t err_index;       /* original-numbering face/cell index of the first failure, or -1 */
    int64_t n_rho_floor;     /* cells where rho < 1e-7 was reset (Setka_physics.cpp:1784-1794) */
    int64_t n_p_floor;       /* cells where p < 1e-8 was reset (Setka_physics.cpp:1981-2001) */
    int32_t status;          /* titan_status of the step loop */
    int32_t err_kind;        /* 0, 11-14 solver region/branch, 15-18 exact HP solver (negative pressure,
                                Newton / bisection without convergence, no wave pattern), 19 non-finite
                                or subnormal contact speed of an HP face (surface tracking), 20
                                non-finite density, 21 a staged cell update's copy wait ran out */
    double  dt_next;         /* CFL dt that the next step will use */
    double  t;               /* accumulated physical time */
    double  gpu_ms;          /* device time of this call's step loop (CUDA events) */
} titan_step_info;

typedef struct titan_ctx titan_ctx;

const char* titan_version(void);
/* Message of the last failing call on this thread. */
const char* titan_last_error(void);

/* Validates and uploads the mesh: space-filling-curve renumbering of cells,
 * faces and nodes (bit-exact and invertible), device geometry of layer 0. */
int titan_create(const titan_mesh* mesh, const titan_params* params, titan_ctx** out);
int titan_destroy(titan_ctx* ctx);

/* Per-face solver choice (Gran::Get_method, TITAN/source/Gran.cpp:3-14) as
 * data: n_state per face in original numbering. */
int titan_set_face_method(titan_ctx* ctx, const int8_t* n_state);

/* Surface-tracking node motion, in place of the prescribed radial law of a
 * context created with move = 1: Setka::Culc_Velocity_surface
 * (TITAN/source/Setka_move.cpp:111-1358) and Luch::dvigenie (Luch.cpp:6-739),
 * called from Setka::Go at Setka_physics.cpp:1616-1627. Every step, before its
 * face loop, the faces of each moving surface (face_surf 1 = TS, 2 = HP,
 * 3 = BS; HP faces with fewer than four surface neighbours are skipped) solve
 * their Riemann problem at w = 0 on the step's state; each surface node moves
 * along its direction (x / |x|; with hp_tail, (0, y, z) for an HP node with
 * x < 0) by dt times the mean of velocity_X * ds * n over its
 * faces (ds = dsl on TS, dsc on HP, dsr on BS; with bn_in_p_on_hp the HP
 * faces use the exact gas-dynamic solver). The other nodes of each ray keep
 * their fraction of the segment between the surface nodes and the ray's
 * ends, on the ray's direction. rays: nray x ray_len node ids (original
 * numbering) from the inner end, a shorter ray padded with -1 after its last
 * node; no node on two rays; radii and directions are taken from the current
 * nodes. Smoothing (each adds one more term to a node's mean velocity,
 * Setka_move.cpp:454-1211): on TS and HP, with sglag_TS / sglag_HP, a node
 * moves toward the sphere that best fits it and its surface neighbours,
 * velocity_X * k_sphere * (B2 - x) / dt, B2 = c + (mean |x_j - c| / |x - c|)
 * (x - c); the centre c is fitted when this function is called (the reference
 * refits between Go calls, TITAN/source/TITAN.cpp:109-124; call this again to
 * refit); on BS, with sglag_BS, toward the mean of itself and its neighbours,
 * velocity_BS * sglag_BS_k * (mean - x) / dt, for nodes with more than five
 * neighbours. The reference's head-region limit on the HP sphere term and its
 * smoothing along its own ray families are not applied. params NULL returns
 * to the prescribed motion. */
typedef struct titan_surface_params {
    double velocity_TS, velocity_HP, velocity_BS; /* Phys_param::velocity_TS / _HP / _BS */
    int32_t move_TS, move_HP, move_BS;            /* Phys_param::move_TS / _HP / _BS */
    int32_t null_bn_on_HP;                        /* Phys_param::null_bn_on_HP: the HP cells and face
                                                     states lose their normal B first */
    int32_t sglag_TS, sglag_HP, sglag_BS;         /* Phys_param::sglag_*: surface smoothing (above) */
    int32_t hp_tail;                              /* 1: HP nodes with x < 0 move along (0, y, z) instead
                                                     of x / |x|, the reference's rule for its heliotail
                                                     (Setka_move.cpp:1237-1247) */
    double sglag_TS_k_sphere, sglag_HP_k_sphere;  /* Phys_param::sglag_TS_k_sphere / sglag_HP_k_sphere */
    double sglag_BS_k;                            /* Phys_param::sglag_BS_k */
} titan_surface_params;

int titan_set_surface_motion(titan_ctx* ctx, const titan_surface_params* params, int64_t nray, int32_t ray_len,
                             const int32_t* ray_nodes);

/* The A_Luch spacing law of Luch::dvigenie (TITAN/source/Luch.cpp:9-152) for
 * the rays given to titan_set_surface_motion, in place of the fraction rule:
 * every ray has M0 + M1 + M2 + M3 + M4 + 5 nodes, from the inner end: M0 at
 * R0 + j (R1 - R0) / M0; the R1 node (left where it is); M1 evenly between R1
 * and the TS node (slot M0 + M1 + 1); M11 after the TS at the same step; M2 -
 * M11 up to the HP node (slot M0 + M1 + M2 + 2) by the cubic law of da1, da2;
 * M3 up to the BS node (slot M0 + M1 + M2 + M3 + 3) by the law of da3, da4;
 * M4 up to the end, placed at R5, by the law of da5. The TS, HP and BS radii
 * are those of the ray's surface nodes after they have moved in the step.
 * Geo_param's names (TITAN/source/Geo_param.h:22-63); one set for all rays
 * (the reference's per-ray da1..da5 overrides are not taken). NULL returns to
 * the fraction rule; titan_set_surface_motion clears the law. */
typedef struct titan_ray_law {
    int32_t M0, M1, M11, M2, M3, M4;
    int32_t pad[2];
    double R0, R1, R5;
    double da1, da2, da3, da4, da5;
} titan_ray_law;
int titan_set_ray_law(titan_ctx* ctx, const titan_ray_law* law);

/* Halo exchange of a sharded step (several contexts, one per GPU, each on the
 * cells one rank owns plus a layer of copies of its neighbours' cells; no
 * reference counterpart: the reference runs one OpenMP process per mesh).
 * send_ids: this context's cells that other ranks keep copies of; recv_ids:
 * its copies, both in the context's original numbering and in the order the
 * peers agree on. titan_pack_halo writes the send cells' states, whole cells
 * of 8 + npassive doubles each ([n_send][ns]), to a DEVICE buffer on this
 * context's GPU; titan_unpack_halo writes a device buffer of the same form
 * into the copies. Both are ordered on titan_stream(ctx) and return without
 * waiting: work on another stream that reads a packed buffer, or writes one
 * to be unpacked, orders itself against this stream (an event, or the
 * stream itself as the exchange's stream). */
int titan_set_halo(titan_ctx* ctx, int64_t n_send, const int32_t* send_ids, int64_t n_recv, const int32_t* recv_ids);
/* Faces (original numbering, 1 = left out) whose CFL candidate does not enter
 * dt: on a sharded rank, the faces between two halo cells, whose stencils can
 * reach past the halo (their true candidates come from the rank that owns a
 * side). NULL: every interior face counts, as in Setka::Go. */
int titan_set_cfl_faces(titan_ctx* ctx, const int8_t* exclude);
int titan_pack_halo(titan_ctx* ctx, double* out_device);
int titan_unpack_halo(titan_ctx* ctx, const double* in_device);

/* Cell::parameters[now] for all cells, SoA [TITAN_NV][ncell], original order.
 * Only the rows the context carries (8 + npassive) travel: the download leaves
 * the others as the caller has them, as the reference's step leaves the
 * parameters it does not evolve. */
int titan_upload_state(titan_ctx* ctx, const double* state);
int titan_download_state(titan_ctx* ctx, double* state);

/* Frozen neutral fluids for the Bera sources: SoA [5*nh][ncell] with
 * rho_Hk, Vx_Hk, Vy_Hk, Vz_Hk, p_Hk for k = 1..nh. */
int titan_upload_hfluids(titan_ctx* ctx, const double* h);

/* External plasma sources SoA [4][ncell] (m_x, m_y, m_z, E; the closure or a
 * Monte-Carlo table). They replace the Bera sources; NULL switches back. */
int titan_set_sources(titan_ctx* ctx, const double* src);

/* `nsteps` steps of the plasma loop of Setka::Go. dt_inout: in, dt of the
 * first step (the reference starts with 1e-5); out, the CFL dt of the next
 * step. t_inout: accumulated physical time (drives the node motion). */
int titan_step(titan_ctx* ctx, int64_t nsteps, double* dt_inout, double* t_inout, titan_step_info* info);

/* The same loop paced by the device, for a mesh split over GPUs (no
 * reference counterpart: the reference steps one mesh in one process). All
 * four calls are ordered on titan_stream(ctx) and only titan_get_clock waits
 * for it, so a caller can put its own work (an NCCL exchange of halo cells,
 * an all-reduce of dt) on the same stream between steps without the host
 * taking part:
 *   titan_set_clock   the device clock of a run: dt of the next step, t, and
 *                     cleared counters and error word (as titan_step does
 *                     from dt_inout / t_inout);
 *   titan_step_async  enqueues nsteps steps from the device clock; each step
 *                     leaves its CFL minimum as the next step's dt;
 *   titan_dt_copy     copies the clock's dt to (into_clock = 0) or from (1)
 *                     one double of device memory, e.g. the buffer of an
 *                     all-reduce(min) over the ranks;
 *   titan_get_clock   waits for the stream and reports dt, t and the run's
 *                     status as titan_step does (info may be NULL).
 * titan_pack_halo / titan_unpack_halo are ordered on the same stream too. */
int titan_set_clock(titan_ctx* ctx, double dt, double t);
int titan_step_async(titan_ctx* ctx, int64_t nsteps);
int titan_dt_copy(titan_ctx* ctx, double* dt_device, int32_t into_clock);
int titan_get_clock(titan_ctx* ctx, double* dt, double* t, titan_step_info* info);

/* Node coordinates [nnode*3] (original numbering) for the current layer; the
 * layer's geometry (and the second-order neighbours of a tvd context) is formed
 * again from them, as Setka::Download_cell_parameters followed by
 * Calculating_measure and Init_TVD does (TITAN/source/TITAN.cpp:36-55). */
int titan_upload_nodes(titan_ctx* ctx, const double* xyz);

/* Cell-parameter checkpoints in the reference's binary layout
 * (Setka::Save_cell_parameters / Download_cell_parameters,
 * TITAN/source/Setka_physics.cpp:4108-4231): per cell a count and key/value
 * pairs, then an optional node block. Host-only, no context needed.
 * read: fills state [TITAN_NV][ncell] for the keys rho, Vx, Vy, Vz, p, Bx, By,
 * Bz, Q, rho_He that the file holds (others are skipped; absent ones leave the
 * caller's values); fields_found: bit k set when field k occurred; xyz
 * [nnode*3] (may be NULL) receives the node block when the file has one
 * (has_nodes = 1). write: the first nfields fields per cell, and the node
 * block when xyz is not NULL. */
int titan_read_cell_parameters(const char* path, int64_t ncell, int64_t nnode, double* state, double* xyz,
                               int32_t* fields_found, int32_t* has_nodes);
int titan_write_cell_parameters(const char* path, int64_t ncell, int32_t nfields, const double* state, int64_t nnode,
                                const double* xyz);

/* Node coordinates [nnode*3] and geometry of the current layer (original numbering). */
int titan_download_nodes(titan_ctx* ctx, double* xyz);
int titan_download_geometry(titan_ctx* ctx, double* cell_center, double* cell_volume, double* face_center,
                            double* face_normal, double* face_area);

/* Face fluxes of the last step [nface*11], original numbering: Prho, PVx, PVy,
 * PVz, Pp (energy), PBx, PBy, PBz, PdivB, PQ, Prho_He — the Gran::parameters
 * "P*" values of Culc_Gran_Potok (flux times area). */
int titan_download_face_fluxes(titan_ctx* ctx, double* flux);

/* The space-filling-curve renumbering titan_create applies, computed on the
 * host alone (no device needed): new index -> original index for cells, faces
 * and nodes. No reference counterpart: Setka::Renumerate
 * (TITAN/source/Setka.cpp:443-465) numbers objects in construction order. */
int titan_sfc_renumber(int64_t nnode, int64_t ncell, int64_t nface, const double* node_xyz,
                       const int32_t* cell_nodes, const int32_t* face_cells, int32_t* cell_new2old,
                       int32_t* face_new2old, int32_t* node_new2old);

/* Second-order neighbours of every face (tvd contexts): out [nface*2] =
 * (AA, BB) in original numbering, -1 when absent — Gran::cells_TVD as
 * Setka::Init_TVD (TITAN/source/Setka_physics.cpp:646-738) chooses them on
 * the geometry at titan_create. */
int titan_get_tvd_neighbours(titan_ctx* ctx, int32_t* out);

/* Permutations chosen at upload: new index -> original index. */
int titan_get_permutation(titan_ctx* ctx, int32_t* cell_new2old, int32_t* face_new2old, int32_t* node_new2old);

/* Stateless batch of Phys_param::chlld calls on the device, host buffers.
 * q1/q2 [n*8] (rho,u,v,w,p,Bx,By,Bz), nrm [n*3], w [n], n_state [n].
 * flags: bit0 null_bn, bit1 left_ydar, bit2 contact, bits 4-5 n_disc.
 * precision 64 or 32. Outputs flux [n*8], ds [n*3] = (dsl, dsc, dsr), rc [n]. */
int titan_riemann_batch(int64_t n, const int8_t* n_state, const double* nrm, const double* w, const double* q1,
                        const double* q2, int32_t flags, int32_t precision, double gamma, double* flux,
                        double* ds, int32_t* rc);

/* Stateless batch of Phys_param::Godunov_Solver_Alexashov calls (the exact
 * gas-dynamic solver of HP faces, Phys_param.cpp:1938-2385) on the device,
 * host buffers. nrm [n*3], w [n], q1/q2 [n*5] (rho, u, v, w, p), contact [n]
 * (0/1). Outputs flux [n*5] (mass, momentum, energy), ds [n*3] = (dsl, dsc,
 * dsr), rc [n]: 0, or 1-4 where the reference would exit (negative pressure
 * in Newton, Newton / bisection without convergence, no wave pattern). */
int titan_godunov_batch(int64_t n, const double* nrm, const double* w, const double* q1, const double* q2,
                        const int8_t* contact, double gamma, double* flux, double* ds, int32_t* rc);

/* Monte-Carlo neutral hydrogen through the current plasma state: the source
 * generator the closure is trained on. Physics of the reference's
 * Setka::MK_fly_immit (TITAN/source/Setka_MK.cpp:1752-2314: charge-exchange
 * rate from Velosity_1 :40-50, new velocity by M_K_Change_Velosity :2788-2852),
 * with momentum and energy exchange tallies the reference does not keep
 * (it tallies densities only, Cell.cpp:1042-1085). Neutrals enter through the
 * boundary faces whose Type_Gran bit is set in `face_types`, from a drifting
 * Maxwellian exp(-|v - u_H|^2 / cp_H^2) of density n_H, in proportion to each
 * face's inflow flux. out [5][ncell], original numbering: n_H, then the plasma
 * momentum (3) and energy sources per unit time and volume (the plasma mass
 * source of charge exchange is identically zero). out NULL keeps the result on
 * the device only (for titan_closure_fallback_from_mc). The inflow split, the
 * tracing and the tallies all run on the device; a pass is reproducible for a
 * seed up to the order of the floating-point tally additions. */
typedef struct titan_mc_params {
    double n_H;
    double u_H[3];
    double cp_H;
    int64_t n_particles;
    uint64_t seed;
    int32_t max_cells;   /* cell visits before a particle counts as lost (0: 1000000) */
    int32_t face_types;  /* e.g. (1 << TITAN_FACE_OUTER_HARD) | (1 << TITAN_FACE_OUTER_SOFT) */
    double* trace_out;   /* NULL, or host [n_particles][8]: each neutral's end — position (3),
                            velocity (3), charge exchanges, 4 * cell visits + end kind (0 left
                            through the boundary, 1 lost after max_cells, 2 no outgoing face,
                            3 stopped on a tallied face, titan_set_mc_face_tally) */
} titan_mc_params;

typedef struct titan_mc_info {
    int64_t particles, lost;
    double inflow_rate;  /* neutrals entering per unit time */
    double gpu_ms;
} titan_mc_info;

int titan_mc_sources(titan_ctx* ctx, const titan_mc_params* params, double* out, titan_mc_info* info);

/* Tabulated velocity distributions of the neutrals entering through chosen
 * faces, the reference's face AMR functions (AMR_f, TITAN/source/AMR_f.h)
 * as Monte-Carlo input: Setka::MK_go (TITAN/source/Setka_MK.cpp:1225-1575)
 * launches the neutrals of an interface face from its AMR_f, where the
 * others (and these faces without a table) take the drifting Maxwellian.
 * Each face gives the frame of its AMR_f (Vn, Vt, Vm: a velocity with local
 * coordinates (x, y, z) is x Vn + y Vt + z Vm, Vn pointing into the cell the
 * neutrals enter) and its leaf cells in the reference's tree order, each a
 * box [xL, xR] x [yL, yR] x [zL, zR] of local velocities (0 <= xL < xR) with
 * the distribution's value f. A face's inflow is the sum over its leaves of
 * box volume * f * |box centre x| times the face area (AMR_f::Culk_SpotokV,
 * AMR_f.cpp:4-48), and it joins the other faces' inflow in one CDF. A neutral
 * that starts on such a face takes a leaf by that weight (AMR_f::
 * Get_random_velosity, AMR_f.cpp:50-96) and, in it, x = sqrt(xL^2 + r (xR^2 -
 * xL^2)), y and z uniform (AMR_cell::Get_random_velosity_in_cell,
 * AMR_cell.cpp:273-326). side: 0 the neutrals enter cells[0], 1 cells[1]
 * (interior faces only). Kept by the context for the passes that follow; NULL
 * (or nface = 0) removes the tables. The reference's per-face particle counts
 * (N_particle and weight mu per face) are replaced by one stratified draw of
 * all neutrals over the joint CDF, each with the same weight. */
typedef struct titan_mc_face_dist {
    int64_t nface;
    const int32_t* face;      /* [nface] original face ids, each at most once */
    const int8_t* side;       /* [nface] */
    const double* frame;      /* [nface][9] Vn, Vt, Vm */
    const int64_t* leaf_ptr;  /* [nface + 1] leaves of face i: leaf_ptr[i] .. leaf_ptr[i+1]-1 */
    const double* leaf_box;   /* [nleaf][6] xL, xR, yL, yR, zL, zR */
    const double* leaf_f;     /* [nleaf] */
} titan_mc_face_dist;
int titan_set_mc_face_dist(titan_ctx* ctx, const titan_mc_face_dist* dist);

/* Outgoing velocity distributions tallied on chosen faces, the other half of
 * the reference's face AMR coupling: a neutral that reaches a listed face
 * from its side cell (side 0: leaving cells[0]; 1: leaving cells[1]) stops
 * there (Setka_MK.cpp:2165-2182) and AMR_f::Add_particle (AMR_f.cpp:240-316)
 * adds mu / |v . Vn|, mu and mu / (v . Vn)^2 to the face's moments n, Smu,
 * nn, and mu to the first leaf (half-open boxes, in the given order) holding
 * its local velocity (x, y, z) = (v . Vn, v . Vt, v . Vm), clamped 1e-7
 * inside the leaves' bounding box (a velocity no leaf holds shrinks toward
 * the origin by 0.995 per try, at most 30 tries, else it counts as
 * unplaced). After each pass the moments are per unit face area and each
 * leaf's weight per unit box volume, face area and box-centre x
 * (AMR_f::Normir_velocity_volume, AMR_f.cpp:318-336), so a face's tallied
 * leaves are a table titan_set_mc_face_dist takes for the zone beyond it.
 * Vn points out of the side cell; leaves 0 <= xL < xR. Kept by the context
 * for the passes that follow; NULL removes the tallies. The trace's end kind
 * of such a neutral is 3. */
typedef struct titan_mc_face_tally {
    int64_t nface;
    const int32_t* face;      /* [nface] original face ids, each at most once */
    const int8_t* side;       /* [nface] */
    const double* frame;      /* [nface][9] Vn, Vt, Vm */
    const int64_t* leaf_ptr;  /* [nface + 1] */
    const double* leaf_box;   /* [nleaf][6] xL, xR, yL, yR, zL, zR */
} titan_mc_face_tally;
int titan_set_mc_face_tally(titan_ctx* ctx, const titan_mc_face_tally* tally);
/* The last pass's tallies: leaf_f [nleaf], moments [nface][3] (n, Smu, nn);
 * either may be NULL. unplaced: neutrals no leaf held. */
int titan_get_mc_face_tally(titan_ctx* ctx, double* leaf_f, double* moments, int64_t* unplaced);

/* ---------------------------------------------------------------------------
 * Learned charge-exchange closure (no reference counterpart: it stands in for
 * re-running the Monte-Carlo neutral solver between plasma steps).
 * An MLP 8 -> 128 -> 128 -> 128 -> 128 -> 5 with SiLU, BF16 weights, FP32
 * accumulation; training rounds activations to BF16, inference carries each
 * activation as a BF16 hi + lo pair (about 16 bits) with SiLU in FP32, so the
 * sources are a smooth function of the cell state. Parameters: FP32 masters, TITAN_MLP_NPARAM
 * floats [W1 16x128 | b1 128 | W2 128x128 | b2 | W3 | b3 | W4 | b4 |
 * W5 128x16 | b5 16], W stored [in][out]; inputs 8..15 and outputs 5..15 are
 * padding kept at zero. norm: feature mean[8], 1/std[8], output scale[5].
 * Features and outputs are defined in titan_c-_b200/csrc/closure.h. */
#define TITAN_MLP_NPARAM 53776

typedef struct titan_mlp_train_opts {
    int32_t epochs;
    int32_t batch;     /* rows per Adam step (rows are used in the caller's order) */
    float lr, beta1, beta2;
    float lr_decay;    /* per-epoch factor, 0 = none */
} titan_mlp_train_opts;

/* Inference of X [n][8] (unstandardised features) -> Y [n][5] on the tensor
 * cores (tcgen05, the kernel the step uses). Host buffers. */
int titan_mlp_forward(const float* params, const float* norm, const float* X, int64_t n, float* Y);
/* Loss and gradient of the weighted MSE sum_r rw_r sum_k w_k (Y_rk - T_rk)^2 / n
 * over one batch (BF16 tensor-core GEMMs). w [5] per output; row_w [n] per row
 * (NULL: all 1); Y (may be NULL) receives the outputs. */
int titan_mlp_grad(const float* params, const float* norm, const float* X, const float* T, const float* w,
                   const float* row_w, int64_t n, float* grad, float* loss, float* Y);
/* Adam on the GPU over the same loss; params in/out; loss_per_epoch [epochs]
 * (may be NULL). */
int titan_mlp_train(float* params, const float* norm, const float* X, const float* T, const float* w,
                    const float* row_w, int64_t n, const titan_mlp_train_opts* opts, float* loss_per_epoch);
/* Installs the closure in a context: every step then computes the plasma
 * sources with the network (before the cell update) instead of the Bera
 * formulas or titan_set_sources. params NULL removes it. n_inf / lambda: the
 * cold-model neutral density proxy of the features. */
int titan_set_closure(titan_ctx* ctx, const float* params, const float* norm, double n_inf, double lambda);

/* Training envelope of an installed closure and the sources it falls back
 * on: a cell whose features (closure.h) leave [lo, hi] (8 floats each) takes
 * its sources from src [4][ncell] (original numbering; m_x, m_y, m_z, E; the
 * last Monte-Carlo pass, titan_mc_sources rows 1-4) instead of the network.
 * src NULL keeps the previous table (none: the network everywhere); lo NULL
 * removes envelope and table. titan_closure_outside returns how many cells
 * were outside the envelope in the last step. */
int titan_set_closure_fallback(titan_ctx* ctx, const float* lo, const float* hi, const double* src);

/* The fallback table of titan_set_closure_fallback from the last
 * titan_mc_sources pass of this context (its rows 1-4), copied on the device.
 * Needs an envelope (titan_set_closure_fallback with lo, hi) and a pass. */
int titan_closure_fallback_from_mc(titan_ctx* ctx);
int titan_closure_outside(titan_ctx* ctx, int64_t* n_outside);

/* Launch-shape autotuner (no reference counterpart: the reference's OpenMP
 * loops have no launch shapes). Times every face-flux variant (threads per
 * block x minimum resident blocks per SM) and every cell-update shape on
 * this context's mesh and state, `reps` launches each, and keeps the fastest.
 * Call after titan_upload_state. With a cache file, a line for the same mesh
 * size and step options is reused instead of timing, and new results are
 * appended. The device status is reset, so call it between runs.
 * Face variants 0-6; cell variants 0-5 read each face record from global
 * memory, 6-8 stage the records of a block's faces in shared memory (one bulk
 * copy of the contiguous run its cells own, cp.async for the others) with
 * identical results. A staged shape whose wait for its copy runs out sets
 * err_kind 21 and the step returns TITAN_ETIMEOUT. */
int titan_autotune(titan_ctx* ctx, int32_t reps, const char* cache_path);
int titan_set_tuning(titan_ctx* ctx, int32_t face_variant, int32_t cell_variant);
/* With the closure installed, run its network on a stream of its own beside
 * the face kernel (both read only the step's state; the cell update waits for
 * both), 1, or before it on the context's stream, 0. Results are the same
 * either way. */
int titan_set_closure_overlap(titan_ctx* ctx, int32_t on);
int titan_get_tuning(titan_ctx* ctx, int32_t* face_variant, int32_t* cell_variant, int32_t* face_block,
                     int32_t* face_min_blocks, int32_t* cell_block);

/* The CUDA stream of the context (cudaStream_t), for event timing by callers. */
void* titan_stream(titan_ctx* ctx);

/* Per-kernel timing: when on, titan_step records CUDA events around every
 * kernel (no CUDA graph) and accumulates device milliseconds per kernel. */
int titan_set_profiling(titan_ctx* ctx, int32_t on);
/* Up to `cap` entries: names (static strings), total ms and launch counts. */
int titan_kernel_times(titan_ctx* ctx, const char** names, double* total_ms, int64_t* launches, int32_t cap);

/* Bytes of device memory the context holds. */
int64_t titan_device_bytes(titan_ctx* ctx);

/* ---------------------------------------------------------------------------
 * titan_step_noalloc — one plasma step that allocates nothing.
 *
 * No counterpart in the reference. It exists for callers that cannot call
 * cudaMalloc when they step: a code whose allocator owns all device memory (a
 * framework's caching allocator or a pool sized at start-up), a real-time
 * loop that forbids allocation after initialisation, or an embedding that
 * must not touch the CUDA allocator. They pass device arrays they already own
 * (titan_dev_mesh, the states) and get one step of titan_step's kernels.
 *
 * The step's scratch — the per-face flux buffer and its status word — is a
 * fixed array compiled into the library (about 12.6 MB, present on every GPU
 * that loads the library until the process exits), so at most
 * TITAN_NOALLOC_MAX_FACES faces; larger meshes get TITAN_EINVAL. Stationary
 * meshes only (params->move = 0). The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress) and caches it with the
 * device's current context: make that first call before any stream capture.
 * A device reset (cudaDeviceReset) gives the device a new context; the next
 * call then looks the address up again, so after a reset, too, the first call
 * comes before any capture. All calls share the array, which keeps the
 * previous call's contents (each call resets the status word itself), so calls
 * that overlap on the GPU race; run them one at a time. ncell must satisfy
 * 3 ncell <= nface (6 faces per cell, 2 cells per face); other sizes get
 * TITAN_EINVAL.
 *
 * All pointers in titan_dev_mesh and state_in/state_out are DEVICE memory,
 * in the library's kernel layout, in any consistent cell/face numbering:
 * states SoA [8 + npassive][ncell]; per-face arrays [nface]; [3][n] SoA for
 * vectors; bc_vals SoA [TITAN_NV][nbc]; cell_faces [6][ncell] face ids with
 * bit 31 set where the cell is the face's cells[1]. dt: this step's dt.
 * dt_next (host): the CFL dt of the next step. err_kind (host, may be NULL):
 * the step's failure kind as in titan_step_info. `stream` is a cudaStream_t
 * (NULL: the legacy default stream); the call returns after it synchronises. */
#define TITAN_NOALLOC_MAX_FACES 131072

typedef struct titan_dev_mesh {
    int64_t ncell, nface, nbc;
    const int32_t* face_c0;        /* [nface] cells[0] */
    const int32_t* face_c1;        /* [nface] cells[1], -1 on boundary faces */
    const int8_t*  face_type;      /* [nface] Type_Gran */
    const int8_t*  face_surf;      /* [nface] Type_Gran_surf */
    const int8_t*  face_method;    /* [nface] n_state, read when method_policy = 0 */
    const int32_t* face_bc;        /* [nface] column of bc_vals for hard faces, else -1 */
    const double*  bc_vals;        /* [TITAN_NV][nbc] */
    const int32_t* cell_faces;     /* [6][ncell] */
    const int8_t*  cell_type;      /* [ncell] */
    const uint8_t* cell_tvd;       /* [ncell] */
    const double*  cell_center;    /* [3][ncell] */
    const double*  cell_volume;    /* [ncell] */
    const double*  face_center;    /* [3][nface] */
    const double*  face_normal;    /* [3][nface] unit, from cells[0] to cells[1] */
    const double*  face_area;      /* [nface] */
    const double*  face_half_dist; /* [nface] half the distance between the two cell centres */
    const double*  hfluids;        /* [5*nh][ncell] or NULL when nh = 0 */
} titan_dev_mesh;

int titan_step_noalloc(const titan_dev_mesh* mesh, const titan_params* params, double dt, const double* state_in,
                       double* state_out, double* dt_next, int32_t* err_kind, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TITAN_B200_H */
