/*
 * lbflow.h -- C ABI of the B200 lattice Boltzmann engine (liblbflow_b200.so).
 *
 * The reference crate (gilberto-ribeiro/lbflow, pure Rust, CPU only) has no FFI:
 * its public entry point is `lbflow::solve(momentum::Parameters,
 * Option<Vec<passive_scalar::Parameters>>)` (src/lib.rs:170-191), which builds a
 * `momentum::Lattice` (src/momentum/lattice.rs:27-207), initialises it
 * (src/momentum/lattice.rs:322-328) and loops `main_steps` + residuals + stop
 * (src/momentum.rs:262-293, src/passive_scalar.rs:136-177).  This header splits
 * that monolithic call into the pieces a Rust `extern "C"` facade (or ctypes /
 * cgo / JNI) binds: a domain descriptor that mirrors `momentum::Parameters`,
 * a scalar descriptor that mirrors `passive_scalar::Parameters`, and
 * create / init / step / residual / observe / destroy calls.  Every call returns
 * an lbf_status and never aborts; lbf_last_error() gives the message of the
 * last failure on the calling thread.
 *
 * Conventions
 *  - Node index i = x + nx*(y + ny*z), as in src/momentum/lattice.rs:70-84.
 *  - All host arrays are owned by the caller; the library copies what it needs.
 *    Device memory is owned by the library behind the opaque handles.
 *  - A domain handle is not thread-safe; distinct handles may be used from
 *    distinct threads.
 *  - `stream` arguments are cudaStream_t passed as void* (NULL = legacy stream).
 */
#ifndef LBFLOW_B200_H
#define LBFLOW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBF_ABI_VERSION 1
#define LBF_MAX_SCALARS 4   /* passive scalars one domain advances in its momentum sweep */

typedef enum {
    LBF_OK = 0,
    LBF_EINVAL = 1,      /* bad descriptor or argument (reference: panic!)      */
    LBF_ENOMEM = 2,      /* device or host allocation failed / no room in batch  */
    LBF_EDEVICE = 3,     /* CUDA error                                           */
    LBF_ETIMEOUT = 4,    /* a bounded wait ran out                               */
    LBF_ENAN = 5,        /* non-finite value detected in a reduction             */
    LBF_EUNSUPPORTED = 6,/* valid in the reference model, not built on device    */
    LBF_ESTATE = 7       /* call out of order (e.g. step before init)            */
} lbf_status;

/* velocity_set::VelocitySet discriminants (src/velocity_set.rs:19-25). */
enum { LBF_D2Q5 = 0, LBF_D2Q9 = 1, LBF_D3Q15 = 2, LBF_D3Q19 = 3, LBF_D3Q27 = 4 };

/* BoundaryFace discriminants (src/lib.rs:17-25). */
enum { LBF_WEST = 0, LBF_EAST = 1, LBF_SOUTH = 2, LBF_NORTH = 3, LBF_BOTTOM = 4, LBF_TOP = 5 };

/* CollisionOperator::{BGK(tau), TRT(omega_plus, omega_minus), MRT(rates)} (src/lib.rs:37-42). */
/* LBF_CENTRAL: central-moment collision of the tensor-product sets D2Q9 and D3Q27
 * (no reference counterpart): shear rate 1/tau; relaxation[0] = bulk rate,
 * relaxation[1..4] = rates of the third to sixth orders (values <= 0 mean 1). */
enum { LBF_BGK = 0, LBF_TRT = 1, LBF_MRT = 2, LBF_CENTRAL = 3 };

/* momentum::bc::BoundaryCondition (src/momentum/bc.rs:12-26). */
enum {
    LBF_BC_NO_SLIP = 0,
    LBF_BC_BOUNCE_BACK = 1,      /* moving wall: density, velocity          */
    LBF_BC_ANTI_BOUNCE_BACK = 2, /* pressure: density                       */
    LBF_BC_ZOU_HE = 3,           /* Option<density>, Vec<Option<velocity>>;
                                    D2Q9 as the reference; D3Q19 / D3Q27 velocity
                                    and pressure faces are an extension         */
    LBF_BC_PERIODIC = 4
};

/* passive_scalar::bc::BoundaryCondition (src/passive_scalar/bc.rs:9-29). */
enum {
    LBF_SBC_ANTI_BOUNCE_BACK = 0,     /* Dirichlet: scalar_value             */
    LBF_SBC_ANTI_BB_NO_FLUX = 1,
    LBF_SBC_BB_NO_FLUX = 2,
    LBF_SBC_ZEROTH_ORDER_NO_FLUX = 3, /* unknown_populations_only            */
    LBF_SBC_SECOND_ORDER_NO_FLUX = 4, /* unknown_populations_only            */
    LBF_SBC_PERIODIC = 5
};

/* passive_scalar::bc::InnerBoundaryCondition (src/passive_scalar/bc.rs:31-35). */
enum { LBF_INNER_ANTI_BOUNCE_BACK = 0, LBF_INNER_BOUNCE_BACK = 1 };

/* Population storage on the device.  Collision arithmetic runs in FP64 for
 * LBF_STORE_F64 and in FP32 for the other three.  The *_DEV formats store the
 * deviation f_i - w_i (momentum) in 16 bits. */
enum { LBF_STORE_F64 = 0, LBF_STORE_F32 = 1, LBF_STORE_F16DEV = 2, LBF_STORE_BF16DEV = 3 };

/* LBF_COMPAT_REFERENCE reproduces the reference arithmetic exactly, including
 * its quirks (force only in BGK collision, src/momentum/node.rs:311-333; the MRT
 * equilibrium-moment functions of src/velocity_set/d2q9.rs:247-264 and
 * src/velocity_set/d3q19.rs:550-587).  LBF_COMPAT_PHYSICS adds the Guo source
 * term to TRT/MRT and uses m_eq = M f_eq. */
enum { LBF_COMPAT_REFERENCE = 0, LBF_COMPAT_PHYSICS = 1 };

/* Node class bits returned by lbf_domain_get_node_class (exact-parity masks). */
#define LBF_CLASS_SOLID       0x1u   /* NodeType::Solid (src/lib.rs:31-35)                     */
#define LBF_CLASS_BOUNCE_BACK 0x2u   /* fluid node with a solid neighbour (lattice.rs:177-191) */
#define LBF_CLASS_FACE_SHIFT  2      /* bit 2+f: fluid node on face f (lattice.rs:163-175)     */

typedef struct {
    int32_t kind;                 /* LBF_BGK / LBF_TRT / LBF_MRT / LBF_CENTRAL        */
    int32_t _pad;
    double tau;                   /* BGK(tau)                                         */
    double omega_plus;            /* TRT(omega_plus, omega_minus): relaxation rates   */
    double omega_minus;
    double relaxation[27];        /* MRT(relaxation_vector), length Q                 */
} lbf_collision_desc;

typedef struct {
    int32_t kind;                 /* LBF_BC_*                                         */
    int32_t has_density;          /* ZouHe: Some(density) ; BounceBack/AntiBB: used   */
    double density;
    int32_t has_velocity[3];      /* ZouHe: Some(u_x) ...                             */
    int32_t _pad;
    double velocity[3];           /* BounceBack / ZouHe wall velocity                 */
} lbf_bc_desc;

/* Mirrors momentum::Parameters (src/momentum.rs:22-37).  The force closure is a
 * constant body force; NodeTypes is a uint8 mask (0 fluid, 1 solid, the map.xyz
 * tokens of src/io.rs:88-96); InitialDensity/InitialVelocity are uniform values
 * or per-node arrays. */
typedef struct {
    int32_t velocity_set;         /* LBF_D2Q9 / LBF_D3Q19 / LBF_D3Q27                 */
    int32_t storage;              /* LBF_STORE_*                                      */
    int64_t n[3];                 /* n[2] ignored for 2-D sets                        */
    lbf_collision_desc collision;
    int32_t has_force;            /* Some(force)                                      */
    int32_t compat;               /* LBF_COMPAT_*                                     */
    double force[3];
    lbf_bc_desc bc[6];            /* indexed by face (LBF_WEST..LBF_TOP)              */
    int32_t face_order[6];        /* order in which face BCs run; all zero = W,E,S,N,B,T */
    const uint8_t* node_type;     /* N entries or NULL (= NodeTypes::OnlyFluidNodes)  */
    double initial_density;       /* InitialDensity::Uniform                          */
    double initial_velocity[3];   /* InitialVelocity::Uniform                         */
    const double* initial_density_field;   /* N entries or NULL                       */
    const double* initial_velocity_field;  /* N*D entries ([node][d]) or NULL         */
} lbf_domain_desc;

typedef struct {
    int32_t kind;                 /* LBF_SBC_*                                        */
    int32_t unknown_populations_only;
    double scalar_value;          /* AntiBounceBack { scalar_value }                  */
} lbf_scalar_bc_desc;

/* Mirrors passive_scalar::Parameters (src/passive_scalar.rs:16-25) and
 * adsorption::Parameters with AdsorptionModel::Langmuir
 * (src/passive_scalar/adsorption.rs:4-28). */
typedef struct {
    int32_t velocity_set;
    int32_t inner_boundary_condition;     /* LBF_INNER_*                              */
    lbf_collision_desc collision;
    int32_t has_source;                   /* Some(source_value) (constant)            */
    int32_t has_adsorption;
    double source_value;
    double initial_scalar_value;          /* InitialScalarValue::Uniform              */
    const double* initial_scalar_field;   /* N entries or NULL                        */
    lbf_scalar_bc_desc bc[6];
    double adsorption_rate;               /* k_a                                      */
    double desorption_rate;               /* k_d                                      */
    double q_max;
    double initial_q_ads;
} lbf_scalar_desc;

typedef struct lbf_domain lbf_domain;

/* ---- library ----------------------------------------------------------- */
int32_t     lbf_abi_version(void);
const char* lbf_last_error(void);
/* sizeof() of the descriptor structs, so bindings can check their layouts. */
size_t      lbf_sizeof(int32_t which);   /* 0 domain_desc, 1 scalar_desc, 2 bc_desc, 3 collision_desc */

/* Velocity-set tables as built on the device side (src/velocity_set.rs:28-190):
 * c[q*3], w[q], q_bar[q], q_faces[6*9] (-1 padded), face_normal[6],
 * mrt[q*q], mrt_inverse[q*q].  Any pointer may be NULL. */
lbf_status lbf_velocity_set_tables(int32_t velocity_set, int32_t* d, int32_t* q,
                                   int32_t* c, double* w, int32_t* q_bar,
                                   int32_t* q_faces, int32_t* face_normal,
                                   double* mrt, double* mrt_inverse);

/* ---- one domain (replaces momentum::Lattice + passive_scalar::Lattice) ---- */
/* Lattice::new (src/momentum/lattice.rs:27-207). */
lbf_status lbf_domain_create(const lbf_domain_desc* desc, lbf_domain** out);
/* passive_scalar::Lattice::new (src/passive_scalar/lattice.rs:26-181).  Up to
 * LBF_MAX_SCALARS calls per domain, before lbf_domain_init: the scalars of
 * passive_scalar::LatticeVec (src/passive_scalar/lattice.rs:353-430), numbered in
 * attach order.  One momentum sweep advances all of them: each step updates the
 * momentum populations of a node, then each scalar's in turn.  Scalars interact
 * only through the shared velocity, as in the reference. */
lbf_status lbf_scalar_attach(lbf_domain* dom, const lbf_scalar_desc* desc);
/* Lattice::initialize_nodes (src/momentum/lattice.rs:322-328,
 * src/passive_scalar/lattice.rs:241-246): f = f_eq(rho0, u0) on fluid nodes. */
lbf_status lbf_domain_init(lbf_domain* dom, void* stream);
/* nsteps x main_steps (src/momentum/lattice.rs:431-441 then
 * src/passive_scalar/lattice.rs:342-350), asynchronous on `stream`.  With
 * residual_interval k > 0, the residuals of every step t with t % k == 0 are
 * computed (compute_lattice_residuals, src/momentum/lattice.rs:369-394). */
lbf_status lbf_domain_step(lbf_domain* dom, int64_t nsteps, int64_t residual_interval, void* stream);
/* The driver loop of src/momentum.rs:262-293: step until
 * (t > 10 and all residuals <= tolerance) or t > max_iterations.  Residuals are
 * checked every `residual_interval` steps (1 = the reference).  Writes the number
 * of main_steps executed to *steps_done.  Synchronous. */
lbf_status lbf_domain_run(lbf_domain* dom, int64_t max_iterations, int64_t residual_interval,
                          double tolerance_density, double tolerance_velocity,
                          double tolerance_scalar, int64_t* steps_done, void* stream);
/* Residuals of the last residual step: [density, velocity_x.., scalar_0, scalar_1 ..]
 * (1 + D + number of scalars entries).  Synchronous.  *time_step receives the step
 * they belong to (-1 if none yet). */
lbf_status lbf_domain_residuals(lbf_domain* dom, double* out, int64_t* time_step);
/* Moments at the current time step (what write_data stores in data/<t>/,
 * src/momentum/io.rs:74-192): density[N], velocity[N*D], scalar[N] of scalar 0
 * (host pointers, any may be NULL).  Solid nodes report their initial values. */
lbf_status lbf_domain_get_moments(lbf_domain* dom, double* density, double* velocity,
                                  double* scalar, void* stream);
/* Scalar `index` (attach order) at the current time step, scalar[N] (host pointer;
 * passive_scalar/io.rs write_data of that lattice). */
lbf_status lbf_domain_get_scalar(lbf_domain* dom, int32_t index, double* scalar, void* stream);
/* Adsorbed amount q_ads per node of scalar 0 (0 where not a bounce-back node). Host pointer. */
lbf_status lbf_domain_get_q_ads(lbf_domain* dom, double* q_ads);
/* The same for scalar `index`. */
lbf_status lbf_domain_get_q_ads_at(lbf_domain* dom, int32_t index, double* q_ads);
/* FP64 inventories over fluid nodes: [sum rho, sum rho*u (D), sum C, sum q_ads] (C, q_ads
 * of scalar 0). */
lbf_status lbf_domain_inventory(lbf_domain* dom, double* out, void* stream);
/* Node classes (LBF_CLASS_* bits) and solid-neighbour link masks (bit i: the
 * neighbour along c_i is solid), computed on the device. */
lbf_status lbf_domain_get_node_class(lbf_domain* dom, uint32_t* node_class, uint32_t* links);
/* Launch options (no reference counterpart; used by the autotuner):
 * LBF_OPT_BLOCK_X  threads per block along x for the unstaged sweep (0 = heuristic)
 * LBF_OPT_STAGE    1 = one-shot staging of the pull rows in shared memory with bulk
 *                  copies when the shape allows it (nx <= 512, rows 16-byte aligned).
 * LBF_OPT_PIPE     1 = pipelined bulk-copy sweep on the lean path (faces periodic or
 *                  no-slip, no scalar, rows 16-byte aligned); default 0 (plain loads).
 * LBF_OPT_PIPE_STAGES  ring depth of the pipelined sweep (0 = from the smem budget).
 * LBF_OPT_COMPACT  1 = on the lean path, sweep a list of the fluid nodes (plus solid
 *                  nodes sharing a 32-byte sector with them) instead of the dense
 *                  lattice; default on for FP64 storage and for D3Q27 other than MRT
 *                  (where it is faster); set before lbf_domain_init.  get: 1 when in
 *                  effect.
 * LBF_OPT_Z_BEGIN, LBF_OPT_Z_END  planes [z_begin, z_end) that steps, observation and
 *                  inventories cover (default all); set before lbf_domain_init.  A
 *                  z-slab of a larger lattice sweeps its owned planes and keeps one
 *                  ghost plane on each side (see the halo calls below).
 * LBF_OPT_SPARSE   1 = on the lean path, store the populations of the fluid nodes only
 *                  and sweep them (no solid bytes move, every thread updates a fluid
 *                  node); 0 = dense layout; default: sparse on the lean path when at
 *                  least 5 % of the nodes are solid.  Set before lbf_domain_init.
 *                  get: 1 when in effect.
 * LBF_OPT_STREAMING  streaming scheme of the sparse layout on the lean path:
 *                  LBF_STREAM_PULL (two buffers; each step reads its neighbours'
 *                  slots), LBF_STREAM_PUSH (two buffers; each step reads its own slots
 *                  and writes its neighbours'), LBF_STREAM_INPLACE (AA pattern: one
 *                  buffer; an even step reads and writes each node's own slots, an
 *                  odd step its neighbours').  All three compute the same values bit
 *                  for bit; the in-place scheme needs half the population memory.
 *                  Default (-1): LBF_STREAM_PULL; z-slabs always pull, and so do
 *                  domains with explicit faces or a scalar.  Set before
 *                  lbf_domain_init.  get: the scheme in effect.
 * LBF_OPT_SROUND   16-bit deviation storage: 1 = stochastic rounding of the stored
 *                  values (seeded by node and time step, so runs repeat exactly),
 *                  0 = round to nearest; default 1.
 * LBF_OPT_SEED_OFFSET  node index (in the whole lattice) of this lattice's node 0:
 *                  a z-slab sets it so that its nodes round as in the whole lattice.
 * LBF_OPT_WAIT_LIMIT  polls after which a bounded wait of the staged sweeps (on
 *                  their bulk copies) gives up: the step then returns LBF_ETIMEOUT
 *                  once the copies in flight have landed, and the domain stays
 *                  usable (re-initialise it).  -1 = default (2^22 polls); 0 makes
 *                  every such wait give up at once, to exercise that path.
 * lbf_domain_get_option reports whether STAGE / PIPE are in effect for the domain. */
enum { LBF_OPT_BLOCK_X = 0, LBF_OPT_STAGE = 1, LBF_OPT_PIPE = 2, LBF_OPT_PIPE_STAGES = 3, LBF_OPT_COMPACT = 4,
       LBF_OPT_Z_BEGIN = 5, LBF_OPT_Z_END = 6, LBF_OPT_SPARSE = 7, LBF_OPT_STREAMING = 8, LBF_OPT_SROUND = 9,
       LBF_OPT_WAIT_LIMIT = 10, LBF_OPT_SEED_OFFSET = 11 };
enum { LBF_STREAM_PULL = 0, LBF_STREAM_PUSH = 1, LBF_STREAM_INPLACE = 2 };
lbf_status lbf_domain_set_option(lbf_domain* dom, int32_t option, int64_t value);
lbf_status lbf_domain_get_option(lbf_domain* dom, int32_t option, int64_t* value);
/* Number of main_steps executed so far (the reference's time_step). */
lbf_status lbf_domain_time_step(lbf_domain* dom, int64_t* t);
/* Device bytes held by the domain. */
lbf_status lbf_domain_device_bytes(lbf_domain* dom, int64_t* bytes);
lbf_status lbf_domain_destroy(lbf_domain* dom);

/* ---- checkpoints ----------------------------------------------------------- */
/* No counterpart in the reference, which restarts from the CSV fields of a time
 * step (InitialDensity/InitialVelocity::FromTimeStep, src/momentum/io.rs:358-394):
 * that restores rho and u only, and the populations restart at equilibrium.  A
 * checkpoint holds the domain's whole carried state: the populations (and scalar
 * populations) the next step reads, q_ads and the previous scalar value, the
 * residual moments, the face layers of the previous step, the time step and the
 * last residuals; a run resumed from it continues bit for bit.
 * lbf_domain_checkpoint_bytes: size of the host buffer.  lbf_domain_save copies
 * the state into it.  lbf_domain_load restores it into a domain created from the
 * same descriptors and options and initialised (lattice, storage, layout and
 * scalar set-up are checked: LBF_EINVAL if they differ). */
lbf_status lbf_domain_checkpoint_bytes(lbf_domain* dom, int64_t* bytes);
lbf_status lbf_domain_save(lbf_domain* dom, void* host, int64_t cap, void* stream);
lbf_status lbf_domain_load(lbf_domain* dom, const void* host, int64_t bytes, void* stream);

/* ---- z-slab halos (multi-GPU decomposition) ------------------------------ */
/* No counterpart in the reference (one process, one lattice).  A lattice split
 * into z-slabs across GPUs runs one domain per slab: its owned planes
 * [z_begin, z_end) plus one ghost plane below and above (LBF_OPT_Z_*), with
 * periodic z faces locally.  A ghost plane is either the neighbour's boundary
 * plane (filled by the halo exchange after every step) or solid nodes (a no-slip
 * wall of the whole lattice, folded into the link bits like any solid).  After
 * each step, lbf_domain_halo_pack(face) gathers the populations that leave the
 * owned boundary plane through `face` (LBF_BOTTOM: c_z = -1, LBF_TOP: c_z = +1,
 * ascending direction index) into a contiguous device buffer for the neighbour;
 * lbf_domain_halo_unpack(face) scatters the neighbour's buffer into the ghost plane
 * beyond `face` (the directions the next step pulls from it).  A bottom pack
 * pairs with the lower neighbour's top unpack, and a top pack with the upper
 * neighbour's bottom unpack.  lbf_domain_halo_info gives the number of leaving
 * directions per face, the nodes per plane and the buffer bytes per face.
 * Asynchronous on `stream`. */
lbf_status lbf_domain_halo_info(lbf_domain* dom, int32_t* ndir, int64_t* plane_nodes, int64_t* bytes);
lbf_status lbf_domain_halo_pack(lbf_domain* dom, int32_t face, void* dst, void* stream);
lbf_status lbf_domain_halo_unpack(lbf_domain* dom, int32_t face, const void* src, void* stream);

/* One step of a z-slab domain in two parts, so that the halo exchange overlaps
 * the interior sweep.  Part 0 updates the owned boundary planes (z_begin and
 * z_end - 1); lbf_domain_halo_pack then reads them and lbf_domain_halo_unpack
 * writes the ghost planes that the next step reads, on any stream ordered after
 * part 0.  Part 1 updates the planes between them, evaluates the residuals of a
 * residual step (k as in lbf_domain_step) and ends the step.  Parts 0 and 1
 * alternate (LBF_ESTATE otherwise); other stepping, observing and checkpoint calls
 * wait for part 1.  Same results as lbf_domain_step. */
lbf_status lbf_domain_step_part(lbf_domain* dom, int32_t part, int64_t residual_interval, void* stream);

/* ---- FP64 fluid sums with no device allocation --------------------------- */
/* No counterpart in the reference (whose reductions are rayon sums on the CPU).
 * For callers that cannot allocate device memory when they need the sums: hosts
 * whose HBM is already reserved by their own caching allocator (an allocation
 * behind its back breaks its accounting) or by lattices sized to fill it (an
 * allocation would fail).  Computes [sum rho, sum rho*u_a (d values), sum C, sum q_ads] over the
 * nodes whose node_class lacks LBF_CLASS_SOLID, from caller-owned device arrays
 * (density[n], velocity[n*d], optional scalar[n] and q_ads[n], node_class[n] as
 * returned by lbf_domain_get_node_class), into the caller-owned device array
 * out[3 + d].  Scratch lives in a fixed 16 KiB static device array that every
 * GPU loading the library holds until exit; each call clears it first, and calls
 * that overlap on the GPU race on it.  The first call on a device looks up that
 * array's address (cudaGetSymbolAddress) with the device current and loads the
 * entry point's kernels: make it before any stream capture.  Rejects n > LBF_NOALLOC_MAX_NODES and d outside {2, 3}. */
#define LBF_NOALLOC_MAX_NODES 2147483647LL
lbf_status lbf_inventory_noalloc(const double* density, const double* velocity, const double* scalar,
                                 const double* q_ads, const uint32_t* node_class, int64_t n, int32_t d,
                                 double* out, void* stream);

/* ---- output text (the reference's CSV writers) ---------------------------- */
/* The reference writes every output step as `{:.8e}` CSV text, one node per line
 * (src/momentum/io.rs:112-192, src/passive_scalar/io.rs:76-108), and the node
 * coordinates once (src/momentum/io.rs:194-224).  These host-only calls format
 * that text on `threads` host threads (<= 0: all cores) in Rust's style
 * ("1.00000000e0", "-2.50000000e-5", "NaN", "inf").  lbf_format_csv writes `rows`
 * lines of `cols` comma-separated values taken row-major from `values`;
 * lbf_format_coordinates writes the "i,j[,k],x,y[,z],fluid|solid" rows of an
 * n[0] x n[1] (x n[2]) lattice with node-centred coordinates (i + 0.5) * delta_x
 * (src/momentum/lattice.rs:86-89).  Neither writes a header line.  With out ==
 * NULL they only report the length in *len; otherwise they fail with LBF_EINVAL
 * if cap < *len. */
lbf_status lbf_format_csv(const double* values, int64_t rows, int32_t cols, char* out, int64_t cap,
                          int64_t* len, int32_t threads);
lbf_status lbf_format_coordinates(const int64_t* n, int32_t d, double delta_x, const uint8_t* node_type,
                                  char* out, int64_t cap, int64_t* len, int32_t threads);

/* ---- batches: many domains stepped together (serving) --------------------- */
/* No counterpart in the reference, which solves one case per process.  A batch
 * advances many initialised domains together: the domains of one kernel
 * configuration (velocity set, collision, storage, explicit faces) share one
 * launch per time step, and a chunk of `residual_interval` = k steps plus an
 * on-device residual + stop-rule evaluation is captured once as a CUDA graph and
 * replayed.  Each domain stops exactly where lbf_domain_run(max_iterations, k,
 * tol_*) would stop it, with the same fields.  Domains with scalars, the
 * central-moment collision or the sparse layout with explicit faces run their
 * own single-domain sweep inside the chunk graph: they are admitted only with an
 * even residual_interval and without the pipelined or staged sweep
 * (LBF_EUNSUPPORTED otherwise); z-slab domains are not batched.  While admitted,
 * a domain refuses the standalone
 * calls (LBF_ESTATE); lbf_batch_poll hands it back once it stopped, and
 * lbf_domain_destroy evicts it first.  The batch object is thread-safe.
 *
 * lbf_batch_create: budget_bytes = device bytes the admitted domains may hold
 *   (0: 90 % of the free device memory now).
 * lbf_batch_admit: LBF_ENOMEM when the domain's device bytes do not fit the budget.
 * lbf_batch_step: enqueues nchunks chunks on `stream` (asynchronous).
 * lbf_batch_poll: returns up to `cap` stopped domains with their status
 *   (1 converged, 2 max_iterations, 3 non-finite residual); wait = 0 returns
 *   nothing while the last chunk is still running.
 * lbf_domain_estimate_bytes: an upper bound of the device bytes a domain built
 *   from these descriptors holds after init and a moments read (admission control
 *   before any allocation). */
typedef struct lbf_batch lbf_batch;
lbf_status lbf_domain_estimate_bytes(const lbf_domain_desc* desc, const lbf_scalar_desc* scalar, int64_t* bytes);
lbf_status lbf_batch_create(int64_t budget_bytes, int64_t residual_interval, lbf_batch** out);
lbf_status lbf_batch_admit(lbf_batch* batch, lbf_domain* dom, int64_t max_iterations, double tol_density,
                           double tol_velocity, double tol_scalar);
lbf_status lbf_batch_step(lbf_batch* batch, int64_t nchunks, void* stream);
lbf_status lbf_batch_poll(lbf_batch* batch, lbf_domain** done, int32_t* status, int32_t cap, int32_t* ndone,
                          int32_t wait);
lbf_status lbf_batch_evict(lbf_batch* batch, lbf_domain* dom);
lbf_status lbf_batch_info(lbf_batch* batch, int64_t* running, int64_t* finished, int64_t* bytes, int64_t* budget);
/* Batch options.  LBF_BATCH_OPT_CHUNK_LAUNCH 1: the batched domains of a group
 * advance a whole chunk (the residual interval k > 1) in one cooperative launch
 * over the group's packed block index, with a grid barrier between the steps;
 * 0 (default): one launch per step, both forms inside the chunk's CUDA graph.
 * The results are the same either way; inside a graph the per-step launches
 * measured slightly faster (64 cavities of 64^2: 6.97 M against 6.61 M
 * domain-steps per second). */
enum { LBF_BATCH_OPT_CHUNK_LAUNCH = 0 };
lbf_status lbf_batch_set_option(lbf_batch* batch, int32_t option, int64_t value);
lbf_status lbf_batch_destroy(lbf_batch* batch);

/* ---- whole solve with host buffers (the `lbflow::solve` drop-in) --------- */
/* Creates a domain from `desc` (+ optional scalar), initialises it, runs
 * `nsteps` main_steps and copies the final moments to the host arrays.
 * Host->device and device->host copies are part of the call. */
lbf_status lbf_solve(const lbf_domain_desc* desc, const lbf_scalar_desc* scalar,
                     int64_t nsteps, double* density, double* velocity, double* scalar_out,
                     void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LBFLOW_B200_H */
