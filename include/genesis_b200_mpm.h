/*
 * genesis_b200_mpm.h -- C ABI of the B200-native MLS-MPM substep.
 *
 * The library replaces the gstaichi kernels of Genesis's MPM hot path:
 *   MPMSolver.substep_pre_coupling   genesis/engine/solvers/mpm_solver.py:471-483
 *     (reset_grid_and_grad :540-550, compute_F_tmp :261-267, svd :269-275, p2g :290-389)
 *   LegacyCoupler.couple -> mpm_grid_op   genesis/engine/couplers/legacy_coupler.py:941-954, 352-496
 *   MPMSolver.substep_post_coupling  genesis/engine/solvers/mpm_solver.py:498-509
 *     (g2p :391-449, _is_state_valid :451-457)
 *   MPMSolver state I/O              genesis/engine/solvers/mpm_solver.py:686-741, 803-905
 *
 * Conventions
 *   - Every entry point is extern "C", takes plain pointers and sizes, and returns an
 *     int status: MPM_OK (0) or a negative MPM_E_* code.  Launch/config errors are
 *     reported synchronously; numerical failures (NaN, stencil outside the grid) are
 *     recorded in a device status word read with mpm_status().
 *   - The caller (PyTorch on the Python side) owns all device memory.  The library
 *     borrows pointers for the duration of a call, never allocates, never frees
 *     (except mpm_graph_* which own a cudaGraphExec_t) and never synchronises except
 *     in mpm_status().
 *   - All work is enqueued on the stream passed in (a cudaStream_t as void*; NULL
 *     means the legacy default stream).
 *   - Arithmetic is float32 throughout, as with gs.init(precision="32").
 *
 * Data layout in device memory
 *   particles (sorted by grid block; "slot" order):
 *     state   float[MPM_STATE_CH][state_stride], planar: channel c of slot s is
 *             state[c*state_stride + s].  Channels: x(0..2) v(3..5) C(6..14, row-major)
 *             F(15..23, row-major) Jp(24).
 *     mat     uint8[n]  material index local to the particle's instance
 *     pflags  uint8[n]  bit0 active, bit1 free (non-free particles act as boundary)
 *     gid     int32[n]  original (API-order) global index of the particle in slot s
 *     slot    int32[n]  inverse of gid: slot of the particle with original index i
 *     mu_p, lam_p  float[n] optional per-particle Lame parameters (NULL: use the table)
 *     actu, muscle_dir  optional muscle inputs in API (original) order, read through gid:
 *             float[n] actuation and float[n][3] fibre direction; both or neither
 *   grid: block-major, MPM_BLOCK^3 nodes per block, blocks of instance k start at
 *     instances[k].blk_base; workspace-resident (see mpm_workspace_bytes).
 */
#ifndef GENESIS_B200_MPM_H
#define GENESIS_B200_MPM_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPM_ABI_VERSION 14

#define MPM_OK 0
#define MPM_E_INVALID -1     /* bad argument / inconsistent sizes */
#define MPM_E_CUDA -2        /* a CUDA runtime call failed */
#define MPM_E_CAPACITY -3    /* a size exceeds a compiled-in limit */
#define MPM_E_NOT_SORTED -4  /* p2g/g2p called before the first mpm_sort_particles */

/* device status word bits (mpm_status) */
#define MPM_STATUS_NAN 1u          /* NaN/Inf in particle positions (mpm_solver.py:451-457) */
#define MPM_STATUS_OUT_OF_GRID 2u  /* a stencil node fell outside the grid; contribution skipped */
#define MPM_STATUS_NONFINITE_VEL 4u /* NaN/Inf in a gathered velocity (positions stay clamped) */

#define MPM_STATE_CH 25
#define MPM_CH_X 0
#define MPM_CH_V 3
#define MPM_CH_C 6
#define MPM_CH_F 15
#define MPM_CH_JP 24

#define MPM_BLOCK 4   /* grid block edge in nodes (sort bin and grid-op unit) */

#define MPM_PFLAG_ACTIVE 1u
#define MPM_PFLAG_FREE 2u

/* material kinds (gs.materials.MPM.*) */
#define MPM_MAT_ELASTIC 0        /* materials/MPM/elastic.py */
#define MPM_MAT_ELASTOPLASTIC 1  /* materials/MPM/elasto_plastic.py */
#define MPM_MAT_LIQUID 2         /* materials/MPM/liquid.py */
#define MPM_MAT_SAND 3           /* materials/MPM/sand.py */
#define MPM_MAT_SNOW 4           /* materials/MPM/snow.py */

#define MPM_MATF_NEOHOOKEAN 1    /* Elastic(model="neohooken") */
#define MPM_MATF_VON_MISES 2     /* ElastoPlastic(use_von_mises=True) */
#define MPM_MATF_MUSCLE 4        /* Muscle: Elastic stress + muscle_stiffness * actu * (F_tmp d)(F_tmp d)^T
                                    with fibre direction d (muscle.py:57-65) */

/* problem flags */
#define MPM_PROBF_NONFREE 1      /* some particles are non-free: run the stencil-zeroing pass after p2g */
#define MPM_PROBF_CPIC 2         /* CPIC against the colliders (mpm_particles.cpic_normal/cpic_sep required) */

/* One simulated scene (one environment).  Mirrors the derived constants of
 * MPMSolver.__init__ (mpm_solver.py:31-78) and Simulator (simulator.py:110). */
typedef struct mpm_instance {
    int32_t p_begin;       /* first slot of this instance's particles */
    int32_t p_count;       /* number of particles */
    int32_t res[3];        /* grid_res = upper_cell - lower_cell + 1 */
    int32_t nblk[3];       /* ceil(res / MPM_BLOCK); at most 1023 per axis */
    int32_t lower_cell[3]; /* grid_offset */
    int32_t mat_base;      /* first entry of this instance in the material table */
    int64_t blk_base;      /* first grid block of this instance */
    float dx, inv_dx;
    float dt;              /* substep dt */
    float eps;             /* grid mass threshold gs.EPS (__init__.py:205-206) */
    float gravity[3];
    float bnd_lo[3], bnd_hi[3]; /* CubeBoundary with 3*dx padding (mpm_solver.py:72-78) */
    float stress_scale;    /* -dt * particle_volume * 4 * inv_dx^2 (mpm_solver.py:344) */
    float c_scale;         /* 4 * inv_dx (mpm_solver.py:430) */
    float pad0;
} mpm_instance;

/* One material, resolved per instance. */
typedef struct mpm_material {
    int32_t kind;          /* MPM_MAT_* */
    int32_t flags;         /* MPM_MATF_* */
    float mu, lam;         /* Lame parameters (base.py:61-70; Liquid mu=0 unless viscous) */
    float mass;            /* particle_volume * rho (mpm_solver.py:785) */
    float default_Jp;      /* 1, or 0 for Sand (sand.py:45) */
    float clamp_lo;        /* 1 - yield_lower  (elasto_plastic.py:89, snow.py:67) */
    float clamp_hi;        /* 1 + yield_higher */
    float vm_threshold;    /* von_mises_yield_stress / (2 mu) (elasto_plastic.py:75) */
    float sand_c1;         /* (3 lam + 2 mu) / (2 mu)         (sand.py:67) */
    float sand_alpha;      /* sqrt(2/3) * 2 sin(phi) / (3 - sin(phi)) (sand.py:47-49) */
    float muscle_stiffness; /* Muscle: its Young's modulus (muscle.py:54) */
} mpm_material;

/* Sizes of one problem (one or many instances advanced together). */
typedef struct mpm_problem {
    int32_t n_instances;
    int32_t n_particles;      /* total over instances */
    int64_t n_blocks;         /* total grid blocks over instances */
    int32_t n_materials;      /* total material-table entries */
    int32_t chunk_particles;  /* particles per p2g/g2p work item (64..1024, multiple of 32) */
    int32_t max_chunks;       /* capacity of the chunk table (mpm_max_chunks) */
    int32_t grid_ctas;        /* persistent CTAs for p2g/g2p/grid-op (0: library default) */
    int32_t flags;            /* MPM_PROBF_* */
} mpm_problem;

typedef struct mpm_particles {
    float* state;
    int64_t state_stride;
    uint8_t* mat;
    uint8_t* pflags;
    int32_t* gid;
    int32_t* slot;
    float* mu_p;   /* optional */
    float* lam_p;  /* optional */
    const float* actu;        /* optional, float[n] in API order: actuation (mpm_solver.py:91, 922-934) */
    const float* muscle_dir;  /* optional, float[n][3] in API order: fibre direction (mpm_solver.py:108) */
    /* CPIC (MPM_PROBF_CPIC; mpm_solver.py:357-379, 412-427, legacy_coupler.py:498-525),
     * both zero-initialised by the caller:
     *   cpic_normal  float[n_colliders * 3][state_stride], indexed by API particle id: the
     *                collider-side normal each particle remembers (mpm_rigid_normal);
     *   cpic_sep     uint32[7][state_stride], indexed by slot: byte j < 27 of a particle's
     *                7 words is 1 + the collider separating it from stencil node j in the last
     *                p2g (0: none), byte 27 is nonzero if any is. */
    float* cpic_normal;
    uint32_t* cpic_sep;
} mpm_particles;

/* Kinematic rigid collider coupled in the grid op (legacy_coupler.py:131-343, 385-397):
 * a grid node with mass within its influence = min(exp(-sd / softness), 1) > 0.1 has its
 * velocity relative to the collider's projected (friction, restitution), exactly as
 * _func_collide_in_rigid_geom does; the momentum change is reported back as a force and a
 * torque about `pos` (the reference hands it to its rigid solver).  The pose advances
 * with lin_vel / ang_vel by the instance's dt after every grid op (constant-velocity
 * kinematic motion between host updates). */
#define MPM_COLLIDER_SPHERE 0  /* sd = |p - pos| - data[0]  (utils/sdf_decomp.py:91-92) */
#define MPM_COLLIDER_PLANE 1   /* sd = n . R^T (p - pos), n = data (geom frame, unit) (sdf_decomp.py:94-98) */
#define MPM_COLLIDER_BOX 2     /* half extents data[0..2]; exact box SDF (the reference samples it on a grid:
                                  MPM_COLLIDER_SDF restates that) */

/* Tool entity (engine/entities/tool_entity/mesh.py:80-176, coupled by
 * legacy_coupler.py:346-350 before the rigid geoms): signed distance sampled trilinearly from
 * a voxel grid of the mesh (1 outside the grid), normal by central differences of 1e-2
 * voxel, velocity of the body point from the pose one substep later, friction response
 * (Tool.friction, coup_softness); no restitution and no reaction force.  Its origin moves at
 * lin_vel and stays above `floor` (FloorBoundary.impose_pos, boundaries.py:67-70). */
#define MPM_COLLIDER_TOOL 3

/* Rigid geom through a sampled signed-distance grid, as the reference couples every geom that
 * is not a sphere or a plane (boxes and meshes: utils/sdf_decomp.py:75-276, grids built by
 * rigid_geom.py:147-225): sdf_res3[0] x sdf_res3[1] x sdf_res3[2] values (x-major) at
 * sdf_offset in mpm_tables.sdf_voxels, followed by the same number of gradient triples
 * [n][3] (central differences of 1e-2 cell of the true distance, as _compute_sd_grad takes
 * them).  Voxel coordinate = sdf_scale * (geom-frame point - data) + (sdf_res3 - 1) / 2, data
 * the grid's centre in the geom frame (the centre of the geom's vertex bounds, 0 for a box);
 * inside the grid the distance and the gradient are trilinear; outside it (any coordinate <= 0 or >=
 * res - 1) the proxy |voxel - centre| / sdf_cell + sdf_max and the direction to the centre.
 * Then the same coupling as MPM_COLLIDER_BOX. */
#define MPM_COLLIDER_SDF 4

typedef struct mpm_collider {
    int32_t kind;        /* MPM_COLLIDER_* */
    int32_t instance;    /* instance (environment) it acts on */
    float pos[3];        /* origin of the geom frame, world */
    float rot[9];        /* world-from-geom rotation, row-major */
    float data[3];       /* see MPM_COLLIDER_* */
    float lin_vel[3];    /* velocity of the origin */
    float ang_vel[3];    /* angular velocity, world */
    float friction;      /* coup_friction   (materials/rigid.py:47); Tool.friction (materials/tool.py:10) */
    float softness;      /* coup_softness   (materials/rigid.py:48; materials/tool.py:11) */
    float restitution;   /* coup_restitution (materials/rigid.py:49) */
    int32_t sdf_res;     /* MPM_COLLIDER_TOOL: voxels per axis of its grid */
    int32_t sdf_pad;
    int64_t sdf_offset;  /* MPM_COLLIDER_TOOL: index of its first voxel in mpm_tables.sdf_voxels */
    float sdf_scale[3];  /* voxel coordinate = sdf_scale * (geom-frame point) + (sdf_res - 1) / 2 */
    float floor;         /* MPM_COLLIDER_TOOL: floor height of the tool solver */
    int32_t sdf_res3[3]; /* MPM_COLLIDER_SDF: voxels per axis */
    float sdf_cell;      /* MPM_COLLIDER_SDF: cell size (sdf_cell_size of rigid_geom.py:155-158) */
    float sdf_max;       /* MPM_COLLIDER_SDF: largest sampled distance */
    float sdf_pad2;
} mpm_collider;

/* External force (acceleration) fields of the grid op (engine/force_fields.py; applied per
 * active node after gravity and before the tools, legacy_coupler.py:377-379:
 * v += acc(pos, v) dt for each field in order, each seeing the velocity the previous ones
 * left).  Every field acts on every instance of the problem.  Kinds and the fields they read:
 *   CONSTANT    acc = vec                                             (force_fields.py:49-82)
 *   WIND        acc = vec where |(pos - center) x dir| <= radius, else 0          (:85-144)
 *   POINT       r = pos - vec, d = r / sqrt(|r|^2 + eps); acc = strength d;
 *               acc += (acc - v) flow; acc /= (sqrt(|r|^2 + eps) + 1)^falloff_pow (:147-198)
 *   DRAG        acc = -linear v - quadratic |v| v                                (:201-229)
 *   NOISE       acc = strength (2 u - 1), u uniform in [0, 1)^3 from a counter-based hash of
 *               (seed, node, the problem's grid-op count): the reference draws ti.random, a
 *               stream this does not reproduce                                   (:232-260)
 *   VORTEX      about the z axis through center: r2 = (pos - center).xy, rho = |r2|;
 *               falloff 1 below falloff_min, 1 / (rho - falloff_min + 1)^falloff_pow below
 *               falloff_max, else 0; acc = falloff (strength (-r2.y, r2.x, 0) +
 *               strength2 (-r2.x, -r2.y, 0)) - damping v                         (:263-369)
 *   TURBULENCE  acc = strength (N_x, N_y, N_z)(pos) with N the improved Perlin noise over
 *               three 512-entry permutation tables at perm[perm_offset ...] (x, y, z) at
 *               spatial frequency `frequency`; acc += (acc - v) flow            (:372-540) */
#define MPM_FF_CONSTANT 0
#define MPM_FF_WIND 1
#define MPM_FF_POINT 2
#define MPM_FF_DRAG 3
#define MPM_FF_NOISE 4
#define MPM_FF_VORTEX 5
#define MPM_FF_TURBULENCE 6

typedef struct mpm_force_field {
    int32_t kind;        /* MPM_FF_* */
    int32_t active;      /* ForceField.activate / deactivate: 0 = no effect */
    float vec[3];        /* CONSTANT, WIND: direction * strength; POINT: position */
    float dir[3];        /* WIND: unit direction */
    float center[3];     /* WIND, VORTEX: center */
    float strength;      /* POINT, NOISE, TURBULENCE; VORTEX: strength_perpendicular */
    float strength2;     /* VORTEX: strength_radial */
    float radius;        /* WIND */
    float falloff_pow;   /* POINT, VORTEX */
    float falloff_min;   /* VORTEX */
    float falloff_max;   /* VORTEX (may be +inf) */
    float flow;          /* POINT, TURBULENCE */
    float damping;       /* VORTEX */
    float linear;        /* DRAG */
    float quadratic;     /* DRAG */
    float frequency;     /* TURBULENCE */
    int32_t perm_offset; /* TURBULENCE: first entry of its 3 x 512 permutation tables in perm */
    uint32_t seed;       /* NOISE */
} mpm_force_field;

typedef struct mpm_tables {
    const mpm_instance* instances;  /* device, n_instances entries */
    const mpm_material* materials;  /* device, n_materials entries */
    mpm_collider* colliders;        /* device, n_colliders entries (may be NULL if none) */
    int32_t n_colliders;
    int32_t pad0;
    float* collider_force;          /* device, optional [n_colliders][6]: force xyz, torque xyz;
                                       accumulated (the caller zeroes it) */
    const float* sdf_voxels;        /* device, the voxel grids of the MPM_COLLIDER_TOOL colliders,
                                       each [sdf_res][sdf_res][sdf_res] (x-major) at its sdf_offset */
    const mpm_force_field* force_fields; /* device, n_force_fields entries (may be NULL if none) */
    int32_t n_force_fields;
    int32_t pad1;
    const int32_t* ff_perm;         /* device, the TURBULENCE fields' permutation tables */
} mpm_tables;

/* ---- sizing ------------------------------------------------------------ */

/* ABI version of the loaded library (MPM_ABI_VERSION). */
int mpm_abi_version(void);

/* sizeof(mpm_instance), sizeof(mpm_material), sizeof(mpm_problem), sizeof(mpm_particles),
 * sizeof(mpm_tables), sizeof(mpm_collider), sizeof(mpm_force_field) as compiled into the
 * library, so a binding can verify its mirror of these structs. */
int mpm_struct_sizes(int32_t* out7);

/* Upper bound on the number of p2g/g2p work items for a problem. */
int mpm_max_chunks(int32_t n_particles, int64_t n_blocks, int32_t chunk_particles, int32_t* out);

/* Bytes of device workspace a problem needs: grid momentum/mass and velocity,
 * block flags, active-block list, sort bins, chunk table, permutation scratch and
 * status counters.  The caller allocates it (256-byte aligned) and keeps it for the
 * problem's lifetime. */
int mpm_workspace_bytes(const mpm_problem* prob, uint64_t* out);

/* Byte offsets, inside the workspace, of the grid arrays: momentum+mass as float4
 * (x, y, z, mass) per node and velocity as float4 (x, y, z, z: a copy of z that the
 * packed gather reads as a (z, z) pair), block-major: node
 * (i, j, k) of instance k lives at ((blk_base + ((i/4)*nblk_y + j/4)*nblk_z + k/4) * 64
 * + ((i%4)*4 + j%4)*4 + k%4).  The momentum/mass grid holds p2g's output between
 * mpm_p2g and mpm_grid_op (grid op clears it); velocity holds grid op's output. */
int mpm_grid_offsets(const mpm_problem* prob, uint64_t* mm_offset, uint64_t* vel_offset);

/* Zero the workspace (grid, flags, counters).  Replaces the per-substep
 * reset_grid_and_grad (mpm_solver.py:540-550), which the kernels fold into grid-op. */
int mpm_workspace_init(const mpm_problem* prob, void* workspace, void* stream);

/* ---- hot path ---------------------------------------------------------- */

/* Counting-sort particles by grid block and rebuild the work-item table.  Required
 * before the first p2g; afterwards optional at any interval (stale binning is still
 * correct, only slower).  Permutes every particle array and updates gid/slot. */
int mpm_sort_particles(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par,
                       void* workspace, void* stream);

/* compute_F_tmp + svd + material return mapping + stress + p2g scatter
 * (mpm_solver.py:261-389).  Writes F and Jp of the next frame in place and leaves
 * grid mass/momentum in the workspace.  With MPM_PROBF_CPIC and colliders it first does
 * coupler.preprocess (legacy_coupler.py:498-525: par->cpic_normal) and leaves out, per
 * stencil node, the particles a collider separates from it (mpm_solver.py:357-379,
 * recorded in par->cpic_sep for the g2p that follows). */
int mpm_p2g(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace,
            void* stream);

/* Grid update of LegacyCoupler.mpm_grid_op, MPM core (legacy_coupler.py:364-375, 495-496):
 * momentum -> velocity, gravity, the coupling with tab->colliders (legacy_coupler.py:385-397,
 * reaction into tab->collider_force), CubeBoundary; then the colliders advance by one
 * substep.  Clears mass/momentum after reading. */
int mpm_grid_op(const mpm_problem* prob, const mpm_tables* tab, void* workspace, void* stream);

/* g2p (mpm_solver.py:391-449) with the NaN check of _is_state_valid folded into a
 * device status bit.  Updates x, v, C in place.  With MPM_PROBF_CPIC the nodes p2g
 * recorded as separated contribute the particle's rigid-response velocity instead of the
 * grid's (mpm_solver.py:412-427). */
int mpm_g2p(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace,
            void* stream);

/* g2p of one substep fused with p2g of the next: gathers v, C from the grid velocity of
 * the last grid op, moves x, then updates F/Jp and scatters mass and momentum for the
 * next grid op.  v and C stay in registers (not stored); a later mpm_g2p stores them.
 * Equivalent to mpm_g2p followed by mpm_p2g. */
int mpm_g2p2g(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace,
              void* stream);

/* n_substeps x (p2g, grid_op, g2p); re-sorts before substep i when
 * sort_interval > 0 and (first_substep + i) % sort_interval == 0. */
int mpm_substeps(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace,
                 int32_t n_substeps, int32_t sort_interval, int64_t first_substep, void* stream);

/* Allocation-free mpm_substeps, for callers that cannot allocate device memory: host
 * applications whose own allocator reserves the GPU's memory up front (game engines and
 * simulators that run from a fixed pool), and plugin hosts that forbid their plugins to
 * call cudaMalloc.  The caller still passes the particle buffers and tables; the
 * workspace of mpm_workspace_bytes() is instead a static device array of
 * MPM_NOALLOC_SCRATCH_BYTES (32 MiB) compiled into this library, which every GPU that
 * loads the library holds until the process exits.  Problems whose workspace exceeds it
 * return MPM_E_CAPACITY (a 65^3 grid with 100k particles needs ~22 MiB).  The first call
 * on a device does a one-time set-up: it looks the array's device address up
 * (cudaGetSymbolAddress) with that device current; that first call should come before
 * any stream capture.  Each call clears the bytes it uses and re-bins the particles, so
 * its results match mpm_substeps; all calls share the one array, so calls that overlap
 * on the GPU (other streams, other threads) race and must be serialised by the caller.
 * Outside stream capture every call looks the address up again, so a device reset
 * (cudaDeviceReset) between calls is followed; a call made while `stream` is capturing
 * uses the address an earlier call found, and returns MPM_E_INVALID if there was none.
 * The status word of the run (NaN positions, stencils outside the grid, non-finite
 * velocities) stays in the array until the next call clears it: read it with
 * mpm_noalloc_status.
 * No counterpart in the reference. */
#define MPM_NOALLOC_SCRATCH_BYTES (32u << 20)
int mpm_substeps_noalloc(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par,
                         int32_t n_substeps, int32_t sort_interval, int64_t first_substep, void* stream);

/* The NaN check (mpm_solver.py:505-509, bits of _is_state_valid :451-457) for callers of
 * mpm_substeps_noalloc, who hold no workspace to pass to mpm_status: reads, from the
 * library's static array, the status word that the last mpm_substeps_noalloc call with
 * the same `prob` left, into *out, and, when inst_out is not NULL, the n_instances
 * per-instance words into inst_out (host memory).  With clear != 0 both are reset
 * afterwards.  Synchronises the stream; allocates nothing.  Must be called before the
 * next mpm_substeps_noalloc, which clears them. */
int mpm_noalloc_status(const mpm_problem* prob, int32_t clear, uint32_t* out, uint32_t* inst_out, void* stream);

/* ---- differentiation (every MPM material) -----------------------------------
 * Reverse-mode adjoint of one substep (mpm_solver.py:261-449 with the materials/MPM files: Elastic
 * corotated / neo-Hookean, Muscle, ElastoPlastic von Mises / clamp, Liquid, Sand, Snow;
 * replaces the gstaichi autodiff of substep_post_coupling_grad / couple_grad /
 * substep_pre_coupling_grad, mpm_solver.py:485-517, legacy_coupler.py:996-1017, and its SVD
 * adjoint backward_svd, :1112-1129).  The grid op's colliders are differentiated as the
 * table holds them for this substep (their pose at its start): the tools' responses
 * (tool_entity/mesh.py:147-176) with respect to the node velocity and the tool's position and
 * linear velocity, the rigid geoms' (legacy_coupler.py:297-341) with respect to the node
 * velocity, their pose taken as given; the particle-level coupling (MPM_PROBF_CPIC) with
 * colliders is not differentiated (MPM_E_INVALID).  The colliders are neither moved nor
 * given forces by the call.
 * `state` is the particle state at the START of the substep (unchanged by the call; the
 * particles must still be in the slot order the last mpm_sort_particles produced).
 * `adj` (float[25][state_stride], same planar layout as the state) holds on entry the
 * adjoint of the substep's output x, v, C, F, Jp and on return the adjoint of its input;
 * `lame_bar` (float[3][state_stride]) accumulates per slot dL/dmu, dL/dlam and, when
 * `state->actu` is set (Muscle), dL/dactu (row 2 is untouched otherwise).
 * The caller allocates adj_workspace (mpm_adjoint_workspace_bytes). */
int mpm_adjoint_workspace_bytes(const mpm_problem* prob, uint64_t* out);
int mpm_substep_adjoint(const mpm_problem* prob, const mpm_tables* tab, const mpm_particles* state, float* adj,
                        float* lame_bar, void* workspace, void* adj_workspace, void* stream);
/* mpm_substep_adjoint that also accumulates, into collider_bar (device float[n_colliders][6],
 * zeroed by the caller; may be NULL), dL/d(position) and dL/d(linear velocity) of every tool
 * collider at this substep through this substep's grid op (rows of rigid geoms stay zero).  The
 * chain between substeps (pos' = pos + lin_vel dt, the tool's origin kept above its floor:
 * tool_entity.py:178-191) is the caller's. */
int mpm_substep_adjoint_colliders(const mpm_problem* prob, const mpm_tables* tab, const mpm_particles* state,
                                  float* adj, float* lame_bar, float* collider_bar, void* workspace,
                                  void* adj_workspace, void* stream);

/* Checkpointed reverse pass without a second forward per substep.  The reference's autodiff
 * re-runs the forward of every substep inside its backward (substep_pre_coupling_grad /
 * couple_grad / substep_post_coupling_grad re-evaluate p2g and the grid op before their .grad,
 * mpm_solver.py:485-517, legacy_coupler.py:996-1017); here the recompute of a checkpoint
 * segment records what the adjoint reads, and the adjoint reads it back:
 *   mpm_substeps_record advances the particles by n_substeps substeps (p2g, grid op, g2p per
 *     substep, no re-sort: the particles must be binned by an earlier mpm_sort_particles) and
 *     stores, for substep j, its input state in state_rec[j] (float[25][state_stride], the
 *     state's planar layout) and its grid in the j-th record of grid_rec, each
 *     mpm_record_grid_bytes long: the momentum and mass after p2g and the velocity after the
 *     grid op (float4[n_blocks * 64] planes, written only in the active blocks), then the active
 *     grid blocks the grid op walked (int32 pairs {instance, packed block coordinates}, room for
 *     n_blocks of them) and their number.
 *   mpm_substeps_adjoint_recorded runs the adjoint of recorded substeps first + count - 1 down
 *     to first, as mpm_substep_adjoint would for each (adj and lame_bar as there), reading
 *     state_rec and grid_rec instead of recomputing them; its grid adjoint visits only each
 *     substep's active blocks.
 * Both refuse colliders (MPM_E_INVALID: their poses move between substeps); force fields are
 * allowed.  state_rec holds n_substeps * 25 * state_stride floats, grid_rec n_substeps *
 * mpm_record_grid_bytes bytes.  The particle tables of `par` (mat, pflags, mu_p, lam_p, actu,
 * ...) must be the ones of the recorded run; its state pointer is not read by the adjoint. */
int mpm_record_grid_bytes(const mpm_problem* prob, uint64_t* out);
int mpm_substeps_record(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace,
                        int32_t n_substeps, float* state_rec, void* grid_rec, void* stream);
int mpm_substeps_adjoint_recorded(const mpm_problem* prob, const mpm_tables* tab, const mpm_particles* par,
                                  int32_t first, int32_t count, const float* state_rec, const void* grid_rec,
                                  float* adj, float* lame_bar, void* adj_workspace, void* stream);

/* ---- timing ----------------------------------------------------------------
 * mpm_substeps with a CUDA event recorded on `stream` after every launch group: on return
 * (the stream is synchronised) ms_by_kind[k] holds the device milliseconds spent in kernels
 * of kind k and launches_by_kind[k] their number of kernel launches, both arrays of
 * MPM_N_KINDS entries.  Consecutive events bracket consecutive launches, so the kinds' times
 * add up to the run's device time.  The simulation advances exactly as with mpm_substeps.
 * No counterpart in the reference (its Taichi kernels are timed by its own profiler). */
#define MPM_KIND_SORT 0        /* the 7 kernels of mpm_sort_particles */
#define MPM_KIND_P2G 1
#define MPM_KIND_GRID_OP 2
#define MPM_KIND_G2P 3
#define MPM_KIND_G2P2G 4       /* g2p of one substep fused with p2g of the next */
#define MPM_N_KINDS 5
int mpm_substeps_profile(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace,
                         int32_t n_substeps, int32_t sort_interval, int64_t first_substep, float* ms_by_kind,
                         int32_t* launches_by_kind, void* stream);

/* Read (and optionally clear) the device status word; synchronises the stream. */
int mpm_status(const mpm_problem* prob, void* workspace, int32_t clear, uint32_t* out, void* stream);

/* Enqueue a copy of the device status word into host memory `out` on `stream` and return
 * without waiting (the asynchronous form of the NaN check at mpm_solver.py:505-509).
 * `*out` is valid once the stream has passed this point (event or stream sync); `out`
 * should be pinned, otherwise the copy is synchronous. */
int mpm_status_enqueue(const mpm_problem* prob, void* workspace, uint32_t* out, void* stream);

/* Per-instance status words (n_instances entries, same bits as mpm_status) into host
 * memory `out`; synchronises the stream.  Instances never share grid memory, so a NaN in
 * one instance leaves the others' results untouched and can be handled per instance. */
int mpm_instance_status(const mpm_problem* prob, void* workspace, int32_t clear, uint32_t* out, void* stream);

/* Enqueue the copy of the per-instance status words into host memory `out` (pinned, for the
 * copy to be asynchronous) and, with clear != 0, their reset, on `stream`; returns without
 * waiting.  `out` is valid once the stream has passed this point.  Used by the serving loop
 * to read a tick's statuses while it prepares the next tick. */
int mpm_instance_status_enqueue(const mpm_problem* prob, void* workspace, int32_t clear, uint32_t* out,
                                void* stream);

/* Number of particles handled by the out-of-tile path since the last clear (tuning aid). */
int mpm_fallback_count(const mpm_problem* prob, void* workspace, int32_t clear, uint64_t* out,
                       void* stream);

/* ---- state I/O (API order) ----------------------------------------------
 * Arrays are in original particle order, flattened over instances:
 * pos/vel float[n][3], C/F float[n][9] (row-major), Jp float[n], active uint8[n].
 * Any output pointer may be NULL to skip it. */

/* _kernel_get_state (mpm_solver.py:723-741) */
int mpm_get_state(const mpm_problem* prob, const mpm_particles* par, float* pos, float* vel, float* C,
                  float* F, float* Jp, uint8_t* active, void* stream);

/* _kernel_set_state (mpm_solver.py:691-712) */
int mpm_set_state(const mpm_problem* prob, mpm_particles* par, const float* pos, const float* vel,
                  const float* C, const float* F, const float* Jp, const uint8_t* active, void* stream);

/* _kernel_set_particles_pos (mpm_solver.py:804-822): sets x of the listed particles
 * (original indices) and resets v=0, F=I, C=0, Jp=default_Jp. */
int mpm_set_particles_pos(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par,
                          int32_t n, const int32_t* idx, const float* pos, void* stream);

/* _kernel_set_particles_vel (mpm_solver.py:853-864) */
int mpm_set_particles_vel(const mpm_problem* prob, mpm_particles* par, int32_t n, const int32_t* idx,
                          const float* vel, void* stream);

/* _kernel_set_particles_active (mpm_solver.py:895-905); active uint8 0/1 */
int mpm_set_particles_active(const mpm_problem* prob, mpm_particles* par, int32_t n,
                             const int32_t* idx, const uint8_t* active, void* stream);

/* _kernel_set_particles_free (mpm_solver.py:988-992); free uint8 0/1 */
int mpm_set_particles_free(const mpm_problem* prob, mpm_particles* par, int32_t n, const int32_t* idx,
                           const uint8_t* free_flag, void* stream);

/* ---- render fields (headless output buffers) ----------------------------
 * _kernel_update_render_fields (mpm_solver.py:743-766).  The problem's particles are
 * n_envs environments of n_per_env particles each (API order: env-major).  For every
 * particle i (API order): render_pos[i] = x, or the "nowhere" point (2333333, 6666666,
 * 5201314) when inactive; render_vel[i] = v only when active (left as is otherwise);
 * render_active[i] = active.  For every visual vertex v of every environment e:
 * vvert_pos[e][v] = sum_j support_w[v][j] * x(e * n_per_env + support_idx[v][j]) and
 * vvert_active[e][v] = active of its first support.  support_idx / support_w are
 * int32 / float [n_vverts][n_supports] (per-environment particle indices, computed on
 * the host as particle_entity.py:192-226 does).  Any output pointer may be NULL. */
int mpm_update_render_fields(const mpm_problem* prob, const mpm_particles* par, int32_t n_envs,
                             int32_t n_per_env, float* render_pos, float* render_vel, uint8_t* render_active,
                             int32_t n_vverts, int32_t n_supports, const int32_t* support_idx,
                             const float* support_w, float* vvert_pos, uint8_t* vvert_active, void* stream);

/* ---- tool signed-distance grids ------------------------------------------
 * compute_sdf_data (utils/mesh.py:179-201) for a triangle mesh already normalised as
 * tool_entity/mesh.py:39-51 does: out[(i * res + j) * res + k] = the signed distance of
 * the point (-r + 2 r i / (res - 1), same for j, k) (r = radius, 0.6 in the reference) to
 * the mesh, negative inside.  Distance to the nearest triangle; the sign from the
 * generalised winding number (inside where it exceeds 1/2).  vertices float [n_verts][3],
 * faces int32 [n_faces][3]; out float [res^3], all device. */
int mpm_sdf_voxelize(const float* vertices, int32_t n_verts, const int32_t* faces, int32_t n_faces, int32_t res,
                     float radius, float* out, void* stream);
/* Signed distance of a closed triangle mesh (device vertices [n_verts][3], faces [n_faces][3])
 * at the nodes of an axis-aligned grid: node (i, j, k) at origin + (i, j, k) * step (host
 * float[3] each), res (host int32[3]) nodes per axis, written x-major into out (device,
 * res[0] * res[1] * res[2] floats).  The distance to the nearest triangle, negative where the
 * generalised winding number exceeds 1/2: igl.signed_distance for a closed mesh, as
 * RigidGeom._compute_sd (engine/entities/rigid_entity/rigid_geom.py:247-249) evaluates it on
 * the geom's sampling grid. */
int mpm_sdf_grid(const float* vertices, int32_t n_verts, const int32_t* faces, int32_t n_faces, const float* origin,
                 const float* step, const int32_t* res, float* out, void* stream);

/* ---- CUDA graphs --------------------------------------------------------
 * Capture n_substeps of mpm_substeps into an executable graph (the pointers in
 * prob/tab/par/workspace are baked in and must stay valid). */
int mpm_graph_create(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par,
                     void* workspace, int32_t n_substeps, int32_t sort_interval,
                     int64_t first_substep, void* stream, void** graph_out);
int mpm_graph_launch(void* graph, void* stream);
int mpm_graph_destroy(void* graph);

#ifdef __cplusplus
}
#endif

#endif /* GENESIS_B200_MPM_H */
