/*
 * soil_cuda.h — C ABI of the B200 (sm_100a) substrate hot path of SOIL.
 *
 * The reference (SueHeir/soil, Rust) exposes this path as ECS plugins and
 * resources, not as an FFI.  Every entry point below replaces one reference
 * system or resource accessor; the citation beside it names the reference
 * function (path inside the reference project, file:line) whose behaviour it
 * reproduces.  A Rust host binds these with `extern "C"` declarations of the
 * same names and argument types, linking libsoil_cuda.so from its build.rs.
 *
 * Conventions
 *   - Every function returns an `int` status (soil_status).  Nothing panics or
 *     throws across the ABI; `soil_last_error(ctx)` holds a one-line message
 *     for the last failure on that context.
 *   - A context is externally synchronised: one host thread at a time.  Each
 *     system owns one CUDA stream; device work is stream-ordered and the host
 *     calls that return data synchronise that stream.
 *   - Host arrays of 3-vectors are interleaved `[n][3]` f64, the reference's
 *     `Vec<[f64; 3]>` layout (crates/soil_core/src/atom.rs:406-431).  On the
 *     device every column is structure-of-arrays.
 *   - Boxes are fully periodic (single rank, periodic self-ghosts); a shear
 *     drive makes them triclinic (Lees–Edwards, xy tilt only).
 */
#ifndef SOIL_CUDA_H
#define SOIL_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SOIL_ABI_VERSION 1

typedef enum soil_status {
    SOIL_OK = 0,
    SOIL_ERR_INVALID = 1,   /* bad argument or call order (reference: panic!/expect) */
    SOIL_ERR_CUDA = 2,      /* a CUDA runtime call failed */
    SOIL_ERR_CAPACITY = 3,  /* a size is beyond a fixed limit; state is unchanged */
    SOIL_ERR_OOM = 4,       /* device allocation failed or the HBM budget is exceeded */
    SOIL_ERR_STATE = 5,     /* call not valid in the current state */
    SOIL_ERR_TIMEOUT = 6,   /* a bounded device wait ran out */
    SOIL_ERR_NOT_FOUND = 7, /* unknown column / job id */
    SOIL_ERR_NO_DEVICE = 8  /* no CUDA device, or the device is not sm_100 */
} soil_status;

/* CommState (crates/soil_core/src/lib.rs:86-94). */
typedef enum soil_comm_state {
    SOIL_FULL_REBUILD = 0,
    SOIL_COMMUNICATE_ONLY = 1
} soil_comm_state;

/* AtomData column classes: #[forward], #[reverse], #[zero]
 * (crates/soil_derive/src/lib.rs:47-52, 392-500). */
#define SOIL_COL_FORWARD 1u
#define SOIL_COL_REVERSE 2u
#define SOIL_COL_ZERO 4u

/* Pair-filter precision of the neighbor build. */
#define SOIL_FILTER_FP64 0        /* every candidate tested in FP64 */
#define SOIL_FILTER_FP32_RECHECK 1 /* FP32 reject test with margin, FP64 recheck of the rest */

/* BoundaryType per axis (domain.rs:36-44). */
#define SOIL_BOUNDARY_PERIODIC 0
#define SOIL_BOUNDARY_FIXED 1  /* atoms outside [lo, hi) are removed by pbc */
#define SOIL_BOUNDARY_SHRINK 2 /* bounds follow the atoms' extent each step */

/* Orthogonal deform styles (DeformStyle, soil_deform/src/lib.rs:168-190). */
#define SOIL_DEFORM_NONE 0
#define SOIL_DEFORM_ERATE 1 /* L(t) = L0 (1 + rate dt step), about the centre */
#define SOIL_DEFORM_VEL 2   /* L(t) = L0 + velocity dt step, about the centre */
#define SOIL_DEFORM_FINAL 3 /* linear ramp of [lo, hi] to a target over a stage */

/* Box: [lo, hi) per axis, all axes periodic (DomainConfig, domain.rs:43-78). */
typedef struct soil_box {
    double lo[3];
    double hi[3];
} soil_box;

/* TOML [neighbor] (NeighborConfig, crates/soil_core/src/neighbor.rs:47-80),
 * plus two fields the reference does not have:
 *   additive_skin — an absolute pair skin s.  The caller stores
 *     cutoff_radius = r + s/2, so the pair cutoff (c_i + c_j)*skin_fraction
 *     equals r_i + r_j + s at skin_fraction = 1; the per-atom displacement
 *     budget becomes (skin_fraction-1)*min_c + s/2 and the ghost buffer twice
 *     that.  s = 0 is exactly the reference.
 *   filter — SOIL_FILTER_FP64 or SOIL_FILTER_FP32_RECHECK (same lists). */
typedef struct soil_neigh_cfg {
    double skin_fraction; /* default 1.0 */
    double bin_size;      /* default 1.0 */
    uint64_t every;       /* default 0 (displacement-based only) */
    uint64_t sort_every;  /* default 1000 (0 = disabled) */
    int32_t check;        /* default 1 */
    int32_t newton;       /* default 1 (half list + reverse comm) */
    double additive_skin; /* default 0.0 */
    int32_t filter;       /* default SOIL_FILTER_FP64 */
    int32_t reserved;
} soil_neigh_cfg;

/* Snapshot of a system's counters. */
typedef struct soil_counts {
    uint64_t nlocal;
    uint64_t nghost;
    uint64_t npairs;             /* neighbor_indices.len() */
    uint64_t step;               /* completed timesteps */
    uint64_t rebuilds;           /* neighbor builds so far */
    uint64_t sorts;              /* spatial sorts that ran (permutation applied or identity) */
    uint64_t steps_since_build;  /* Neighbor.steps_since_build */
    uint64_t filter_candidates;  /* pair candidates tested in the last build */
    uint64_t filter_rechecked;   /* of those, re-tested in FP64 (FP32 mode) */
    int32_t comm_state;          /* soil_comm_state */
    int32_t triclinic;
    int32_t bin_count[3];        /* Neighbor.bin_count */
    int32_t nstencil_forward;    /* Neighbor.bin_stencil_forward.len() */
    double ghost_cutoff;         /* Neighbor.ghost_cutoff */
    double max_cutoff;           /* Neighbor.cached_max_cutoff */
    double tilt_xy;              /* Domain.tilt[0] */
} soil_counts;

/* Device pointers handed to a force hook; valid until the next rebuild.
 * Column c, component k of atom i is columns[c][k * stride + i]. */
typedef struct soil_dev_view {
    uint64_t nlocal;
    uint64_t nghost;
    uint64_t npairs;
    uint64_t stride;
    const double* x;
    const double* y;
    const double* z;
    const double* vx;
    const double* vy;
    const double* vz;
    double* fx;
    double* fy;
    double* fz;
    const double* mass;
    const double* inv_mass;
    const double* cutoff_radius;
    const uint32_t* tag;
    const uint32_t* neighbor_offsets; /* nlocal + 1 */
    const uint32_t* neighbor_indices; /* npairs */
    int32_t ncolumns;
    int32_t newton;
    double* const* columns;           /* device array of ncolumns device pointers */
    void* stream;                     /* cudaStream_t the hook must launch on */
    /* For deterministic consumers (include/soil_consumer.cuh): the transposed
     * half list — in_list[in_start[a] .. in_start[a+1]) are the rows that list
     * atom a, ascending — the ghost images' sources and the reverse-comm fold
     * program (fold_list[fold_start[t] .. fold_start[t+1]) are local t's
     * images, ghost index minus nlocal, in fold order). */
    const uint32_t* in_start;         /* nlocal + nghost + 1 */
    const uint32_t* in_list;          /* npairs */
    const int32_t* origin;            /* nlocal + nghost: source atom of each ghost */
    const uint32_t* fold_start;       /* nlocal + 1 */
    const uint32_t* fold_list;        /* nghost */
    /* Local atom each ghost images (ghost index minus nlocal). */
    const uint32_t* ghost_root;       /* nghost */
    /* Persistent per-neighbor slots (soil_sys_enable_slots; include/soil_slots.cuh):
     * local atom i owns slots [i*slot_max, (i+1)*slot_max) of (partner tag,
     * slot_width f64 payload).  The hook reads the last step's slots ("old")
     * and writes this step's ("new"); the library swaps them after the hook.
     * slot_max == 0: no slots. */
    uint32_t slot_max;
    uint32_t slot_width;
    const uint32_t* slot_old_tag;     /* nlocal * slot_max; 0xFFFFFFFF = empty */
    const double* slot_old_val;       /* nlocal * slot_max * slot_width */
    uint32_t* slot_new_tag;
    double* slot_new_val;
} soil_dev_view;

/* Force hook (the device analogue of a Force-phase system, and of the
 * prototype's GpuForce::record, crates/soil_gpu/src/gpu_state.rs:45-55).
 * Called once per step after ghosts are current and forces are zero; it must
 * only enqueue work on view->stream.  Return 0 on success. */
typedef int (*soil_force_fn)(const soil_dev_view* view, void* user);

typedef struct soil_ctx soil_ctx;
typedef struct soil_sys soil_sys;
typedef struct soil_batch soil_batch;

/* ---- lifecycle ---------------------------------------------------------- */
int soil_abi_version(void);
/* Create a context on CUDA device `device`; hbm_budget_bytes = 0 means no cap. */
int soil_ctx_create(int device, uint64_t hbm_budget_bytes, soil_ctx** out);
/* Destroy the systems, batches and servers of a context before the context:
 * their device memory comes from the context's stream-ordered pool, which is
 * released here (memory still allocated from it is returned when freed). */
int soil_ctx_destroy(soil_ctx* ctx);
const char* soil_last_error(const soil_ctx* ctx);
/* Device bytes currently held by all systems of the context. */
int soil_ctx_bytes_in_use(const soil_ctx* ctx, uint64_t* out);
/* Device allocations and frees the context has made so far (no reference
 * counterpart: lets a host check that steady-state steps allocate nothing). */
int soil_ctx_alloc_count(const soil_ctx* ctx, uint64_t* allocs, uint64_t* frees);

/* ---- systems ------------------------------------------------------------ */
/* Domain + Atom + Neighbor + CommTopology resources of one simulation
 * (AtomPlugin atom.rs:609-621, DomainPlugin domain.rs:406-449,
 *  NeighborPlugin neighbor.rs:516-567, CommunicationPlugin comm.rs:157-202).
 * dt = Atom.dt. */
int soil_sys_create(soil_ctx* ctx, const soil_box* box, const soil_neigh_cfg* cfg,
                    double dt, soil_sys** out);
int soil_sys_destroy(soil_sys* sys);

/* register_atom_data! (atom.rs:106-118): one f64 column of `width` values
 * per atom, flags from SOIL_COL_*.  Must precede soil_sys_setup; a duplicate
 * name returns SOIL_ERR_INVALID (the reference panics). */
int soil_sys_register_column(soil_sys* sys, const char* name, int32_t width,
                             uint32_t flags, int32_t* col_out);

/* Append n local atoms (push_test_atom / unpack_atom, atom.rs:561-574,
 * 539-553).  inv_mass = 1/mass.  columns[c] is n*width_c f64 for column c or
 * NULL for zeros; `columns` may be NULL.  Only before soil_sys_setup. */
int soil_sys_add_atoms(soil_sys* sys, uint64_t n, const uint32_t* tag,
                       const uint32_t* type, const double* pos3,
                       const double* vel3, const double* mass,
                       const double* cutoff_radius, const double* const* columns);

/* neighbor_setup (neighbor.rs:604-665) + comm_setup (comm.rs:253-283). */
int soil_sys_setup(soil_sys* sys);

/* [deform] xy = { style = "erate", rate } — Lees–Edwards shear
 * (soil_deform/src/lib.rs:346-420 setup, 559-603 per step). */
int soil_sys_set_shear(soil_sys* sys, double erate);

/* [deform] x/y/z (dim 0/1/2) = { style, ... } — orthogonal box deformation,
 * applied each step before the initial integration (apply_deform,
 * soil_deform/src/lib.rs:468-557); the bounds at setup are the axis' L0.
 *   SOIL_DEFORM_ERATE: a = rate;  SOIL_DEFORM_VEL: a = velocity;
 *   SOIL_DEFORM_FINAL: a, b = target lo, hi; stage_steps = the length of the
 *   run stage the ramp spans (the reference takes it from RunState).
 * Every deforming step rebuilds the neighbor lists.  An axis that reaches
 * zero size makes soil_step fail with SOIL_ERR_INVALID (the reference
 * panics).  Before setup; not for batched systems. */
int soil_sys_set_deform(soil_sys* sys, int32_t dim, int32_t style, double a, double b,
                        uint64_t stage_steps);
/* [deform] remap (default 1): scale local positions with the box about its
 * centre (lib.rs:530-540). */
int soil_sys_set_deform_remap(soil_sys* sys, int32_t remap);
/* [domain] boundary_x/y/z (SOIL_BOUNDARY_*) and shrink_wrap_padding (0: the
 * ghost cutoff), before setup (domain_read_input, domain.rs:460-498).  A
 * non-periodic axis has no ghost images and no comm neighbor: its swaps still
 * pack their face atoms (soil_sys_get_swap_sends) but receive nothing
 * (comm.rs:253-283, 832-835); pbc removes atoms that leave it, last index
 * first by swap-remove (domain.rs:641-662); the displacement check uses the
 * general per-axis path (neighbor.rs:736-756).  Shrink-wrapped axes follow
 * the locals' extent plus the padding every step (shrink_wrap_update,
 * domain.rs:509-575).  Lees–Edwards shear needs periodic x and y (a fixed or
 * shrink-wrapped z works in lamda space, pbc_triclinic domain.rs:673-729);
 * batched systems are periodic. */
int soil_sys_set_boundary(soil_sys* sys, const int32_t type[3], double shrink_padding);
/* Number of atoms swap s packed (its send_indices): recv_count for a swap
 * with a neighbor, the face atoms for one without. */
int soil_sys_get_swap_sends(soil_sys* sys, int32_t s, uint64_t* count);
/* Domain bounds and tilt (xy, xz, yz) as they stand. */
int soil_sys_get_box(soil_sys* sys, double lo[3], double hi[3], double tilt[3]);

/* Built-in consumer: linear repulsion f = k*overlap along the pair normal
 * (docs/src/tutorial/write-your-own-physics.md:56-110) with the radius read
 * from column `radius_col` (a #[forward] width-1 column).  k = 0 disables. */
int soil_sys_set_harmonic(soil_sys* sys, double k, int32_t radius_col);

/* Install (fn != NULL) or remove a force hook; replaces the built-in consumer. */
int soil_sys_set_force_hook(soil_sys* sys, soil_force_fn fn, void* user);

/* Run nsteps full timesteps: every phase below in the reference schedule
 * order (schedule.rs:22-52).  Returns when the work is enqueued and the
 * rebuild decisions are taken; call soil_sys_sync to wait. */
int soil_step(soil_sys* sys, uint64_t nsteps);
int soil_sys_sync(soil_sys* sys);
int soil_sys_stream(soil_sys* sys, void** cuda_stream_out);

/* ---- per-phase systems (each applies its reference run condition) ------- */
int soil_phase_deform(soil_sys* sys);          /* apply_deform       soil_deform/src/lib.rs:435-604 */
int soil_phase_initial(soil_sys* sys);         /* initial_integration soil_verlet/src/lib.rs:131-162 */
int soil_phase_decide_rebuild(soil_sys* sys);  /* decide_rebuild     neighbor.rs:796-822 */
int soil_phase_remove_ghosts(soil_sys* sys);   /* remove_ghost_atoms atom.rs:625-629 */
int soil_phase_zero_forces(soil_sys* sys);     /* zero_all_forces    atom.rs:631-635 */
int soil_phase_shrink_wrap(soil_sys* sys);     /* shrink_wrap        domain.rs:577-589 */
int soil_phase_pbc(soil_sys* sys);             /* pbc / pbc_triclinic domain.rs:611-729 */
int soil_phase_sort(soil_sys* sys);            /* sort_atoms_by_bin  neighbor.rs:834-997 */
int soil_phase_borders(soil_sys* sys);         /* borders            comm.rs:682-860 */
int soil_phase_forward_comm(soil_sys* sys);    /* forward_comm_borders comm.rs:582-592 */
int soil_phase_neighbor(soil_sys* sys);        /* bin_neighbor_list  neighbor.rs:1013-1319 */
int soil_phase_force(soil_sys* sys);           /* Force phase: hook or built-in consumer */
int soil_phase_reverse_comm(soil_sys* sys);    /* reverse_send_force comm.rs:938-1024 */
int soil_phase_final(soil_sys* sys);           /* final_integration  soil_verlet/src/lib.rs:175-194 */

/* ---- read-back (synchronising) ------------------------------------------ */
int soil_sys_counts(soil_sys* sys, soil_counts* out);
/* Atoms [first, first+n) of local+ghost storage; any output may be NULL. */
int soil_sys_get_atoms(soil_sys* sys, uint64_t first, uint64_t n, uint32_t* tag,
                       double* pos3, double* vel3, double* force3,
                       int32_t* image3, int32_t* origin_index);
int soil_sys_get_column(soil_sys* sys, int32_t col, uint64_t first, uint64_t n,
                        double* out /* n*width */);
/* Neighbor.neighbor_offsets (nlocal+1) and neighbor_indices (npairs). */
int soil_sys_get_neighbor(soil_sys* sys, uint32_t* offsets, uint32_t* indices);
/* Number of ghost swaps recorded by the last borders (6 on one rank). */
int soil_sys_num_swaps(soil_sys* sys, int32_t* out);
/* SwapData (comm.rs:114-124) of swap s; send_indices has recv_count entries. */
int soil_sys_get_swap(soil_sys* sys, int32_t s, uint64_t* recv_start,
                      uint64_t* recv_count, double periodic_offset[3],
                      double vel_offset[3], uint32_t* send_indices);
/* Permutation applied by the last spatial sort (perm[new] = old), nlocal entries. */
int soil_sys_get_sort_perm(soil_sys* sys, uint32_t* perm);
/* Device pointers for an external consumer (valid until the next rebuild).
 * Returns after the system's stream has drained, so the pointers may be used
 * on any stream. */
int soil_sys_view(soil_sys* sys, soil_dev_view* out);

/* Persistent per-neighbor state slots: the reference's NeighborSlots
 * (crates/soil_gpu/src/neighbor_slots.rs:19-184: MAX_CONTACTS slots of
 * (partner, payload) per atom, double-buffered, SENTINEL = empty), in FP64
 * and keyed by the partner's TAG instead of its index, so a contact's state
 * survives rebuilds, the spatial sort (an atom's slots move with it) and the
 * pair moving from one atom's CSR row to the other's.  Every local atom gets
 * max_contacts slots of `width` doubles, all empty; the force hook reads and
 * writes them through soil_dev_view (helpers in include/soil_slots.cuh) and
 * the library swaps the two sets after each hook call.  Not for batched
 * systems.  max_contacts in [1, 1024], width in [1, 64]. */
int soil_sys_enable_slots(soil_sys* sys, uint32_t max_contacts, uint32_t width);
/* The slots the last hook call wrote, for local atoms 0..nlocal-1 in their
 * current order: partner_tag (nlocal*max_contacts), payload
 * (nlocal*max_contacts*width). */
int soil_sys_get_slots(soil_sys* sys, uint32_t* partner_tag, double* payload);

/* Checkpoint in the reference's restart wire format: RestartData
 * (soil_print/src/lib.rs:318-418) as write_restart serialises it with bincode 1
 * (soil_print/src/lib.rs:1390-1445): little endian, fixed-width integers, u64
 * length before every Vec, fields in declaration order; the locals only, the
 * registered columns in atom_data_buffers (registration order, each atom's
 * values in a row).  buf NULL: *len gets the size only.  A buffer that is too
 * small returns SOIL_ERR_CAPACITY with *len set.  A pending final half-kick is
 * applied first (the reference writes after FinalIntegration). */
int soil_sys_save_restart(soil_sys* sys, uint64_t total_cycle, uint8_t* buf, uint64_t cap,
                          uint64_t* len);
/* read_restart (soil_print/src/lib.rs:1527-1625): loads a restart into a
 * system with its columns registered and no atoms (before soil_sys_setup):
 * tags, types, positions, velocities, forces, masses, cutoff radii, columns;
 * dt and the step count come from the data. */
int soil_sys_load_restart(soil_sys* sys, const uint8_t* buf, uint64_t len, uint64_t* total_cycle);

/* Stable counting sort of n positions by bin cell that allocates no device
 * memory.  This has no counterpart in the reference: it serves hosts that
 * cannot allocate device memory once they run (a fixed HBM plan, or an
 * allocator that owns the device), giving the same permutation as the
 * spatial sort of soil_phase_sort.  The caller passes device arrays d_x,
 * d_y, d_z (n positions), d_cell (n outputs: the cell of each atom) and
 * d_perm (n outputs: perm[new] = old, stable inside a cell), plus the bin
 * grid (origin, bin_size, bin_count; box_lo, box_size, tilt and triclinic
 * for lamda binning) and a cudaStream_t (NULL = default stream).  Work is
 * enqueued on `stream`.  Scratch is one 16 MiB static device array per GPU,
 * held until process exit; grids above 2,097,152 cells return
 * SOIL_ERR_CAPACITY (bin counts whose product would overflow included).
 * Every call looks up the array's device address (cudaGetSymbolAddress) with
 * the current device; the first call on a device loads the module there, so
 * make that first call before any stream capture.  Calls share the array:
 * calls that overlap on the GPU race and must be serialised.  ctx may be
 * NULL (no message). */
int soil_bin_sort_noalloc(soil_ctx* ctx, const double* d_x, const double* d_y,
                          const double* d_z, uint64_t n, const double origin[3],
                          const double bin_size[3], const int32_t bin_count[3],
                          const double box_lo[3], const double box_size[3],
                          const double tilt[3], int32_t triclinic, uint32_t* d_cell,
                          uint32_t* d_perm, void* stream);

/* ---- batched stepping (many independent systems, one launch per phase) ----
 * The reference steps one system per App; soil_batch steps many set-up
 * systems together, each box through exactly the phases and arithmetic of
 * soil_step, so every system's trajectory, CSR lists, ghost maps and sort
 * permutations are bit-identical to stepping it alone.  Members must use the
 * built-in harmonic consumer (soil_sys_set_harmonic), have no force hook and
 * no SOIL_COL_ZERO column.  While batched, a system's stream is the batch's
 * stream; every soil_sys_* readback stays valid between soil_batch_step calls.
 * Destroying a batched system removes it from its batch first. */
/* Host planning of a step runs per box on a thread pool: SOIL_HOST_THREADS
 * threads (default: hardware threads, at most 16), used when a step plans at
 * least SOIL_HOST_MIN_PARALLEL boxes (default 64). */
int soil_batch_create(soil_ctx* ctx, soil_batch** out);
/* Detaches every member (the systems themselves are not destroyed). */
int soil_batch_destroy(soil_batch* batch);
int soil_batch_add(soil_batch* batch, soil_sys* sys);
int soil_batch_remove(soil_batch* batch, soil_sys* sys);
int soil_batch_size(soil_batch* batch, uint32_t* nsys);
/* nsteps timesteps of every member (final half-kick applied after the last). */
int soil_batch_step(soil_batch* batch, uint64_t nsteps);
int soil_batch_sync(soil_batch* batch);
int soil_batch_stream(soil_batch* batch, void** stream);
/* Stage timers of soil_batch_step (CUDA events on the batch stream):
 * 0 integrate, 1 sort (pbc + spatial sort), 2 borders, 3 neighbor (fold
 * program, forward comm, pair count pass), 4 lists (CSR fill, incoming
 * lists), 5 force (the consumer kernel alone), 6 reverse (reverse comm, final),
 * 7 whole step; the step time minus the stages is time the device waited for
 * the host. */
#define SOIL_BATCH_NUM_TIMERS 8
/* Enables (on != 0) or disables the stage timers; resets every timer sum. */
int soil_batch_set_timing(soil_batch* batch, int32_t on);
int soil_batch_get_timing(soil_batch* batch, double* ms, uint64_t* intervals);
/* Host milliseconds spent planning each part of the step (always measured,
 * reset by soil_batch_set_timing): 0 integrate, 1 sort, 2 border planning,
 * 3 border launches, 4 neighbor, 5 lists + force, 6 waiting for the device. */
#define SOIL_BATCH_NUM_HOST_TIMERS 7
int soil_batch_get_host_timing(soil_batch* batch, double* ms);
/* Batched steps taken, host waits on the device, device bytes of the batch
 * tables, and border passes repeated for a box whose ghosts outgrew its
 * capacity (each repeat grows that box first). */
int soil_batch_stats(soil_batch* batch, uint64_t* steps, uint64_t* host_waits,
                     uint64_t* device_bytes, uint64_t* border_retries);

/* ---- served mode (no reference counterpart: the reference runs one App per
 * process) ------------------------------------------------------------------
 * A request loop on its own host thread admits jobs first come first served
 * while their HBM reservation (natoms * bytes_per_atom + bytes_per_job) fits
 * hbm_budget_bytes and fewer than max_active jobs are resident, keeps every
 * admitted job resident in one soil_batch, advances them together in quanta
 * of at most quantum_steps steps (never past any job's own step count), and
 * retires finished jobs (final state read back, memory freed).  Each job's
 * result is bit-identical to the same system run alone through soil_step.
 * The server's context belongs to the loop thread: do not use it elsewhere
 * while the server exists.  Zero fields take defaults (no budget, 65,536
 * jobs, 50 steps, 1,024 B/atom, 8 MiB/job). */
typedef struct soil_server soil_server;
typedef struct soil_server_cfg {
    uint64_t hbm_budget_bytes;
    uint32_t max_active;
    uint32_t quantum_steps;
    uint32_t bytes_per_atom;
    uint32_t bytes_per_job;
} soil_server_cfg;
/* One job: a periodic box of spheres with the harmonic consumer (radius
 * column #[forward]), optional xy shear, run for `steps` timesteps.  Arrays
 * are copied by soil_server_submit. */
typedef struct soil_job_spec {
    soil_box box;
    soil_neigh_cfg cfg;
    double dt;
    uint64_t natoms;
    const uint32_t* tag;
    const double* pos3;
    const double* vel3;
    const double* mass;
    const double* cutoff_radius;
    const double* radius;
    double harmonic_k;
    double shear_rate;
    uint64_t steps;
} soil_job_spec;
typedef enum soil_job_state {
    SOIL_JOB_QUEUED = 0,
    SOIL_JOB_RUNNING = 1,
    SOIL_JOB_DONE = 2,
    SOIL_JOB_FAILED = 3,
    SOIL_JOB_CANCELLED = 4
} soil_job_state;
/* Times are seconds since the server was created (t_admit, t_done < 0: not yet). */
typedef struct soil_job_info {
    int32_t state;
    uint64_t natoms;
    uint64_t steps;
    uint64_t steps_done;
    double t_submit;
    double t_admit;
    double t_done;
} soil_job_info;
typedef struct soil_server_stats {
    uint64_t queued;
    uint64_t admitted;
    uint64_t completed;
    uint64_t failed;          /* failed or cancelled */
    uint64_t atom_steps;      /* sum over batch steps of resident atoms */
    uint64_t batch_steps;
    double busy_s;            /* host time inside batch steps */
    double elapsed_s;
    uint64_t reserved_bytes;
    int32_t max_active;       /* most jobs resident at once */
} soil_server_stats;
int soil_server_create(soil_ctx* ctx, const soil_server_cfg* cfg, soil_server** out);
/* Stops the loop; queued and resident jobs end as SOIL_JOB_CANCELLED. */
int soil_server_destroy(soil_server* server);
int soil_server_submit(soil_server* server, const soil_job_spec* job, uint64_t* job_id);
int soil_server_poll(soil_server* server, uint64_t job_id, soil_job_info* info);
/* Blocks until the job is done, failed or cancelled (timeout_s < 0: no limit);
 * SOIL_ERR_TIMEOUT when the limit passes first. */
int soil_server_wait(soil_server* server, uint64_t job_id, double timeout_s, soil_job_info* info);
int soil_server_cancel(soil_server* server, uint64_t job_id);
/* Final local atoms of a done job, in the system's final (spatially sorted)
 * order: tags, positions, velocities, image flags; any output may be NULL. */
int soil_server_result(soil_server* server, uint64_t job_id, uint32_t* tag, double* pos3,
                       double* vel3, int32_t* image3);
/* Forgets a finished job (its results included). */
int soil_server_release(soil_server* server, uint64_t job_id);
/* Error message of a failed job. */
int soil_server_job_error(soil_server* server, uint64_t job_id, char* buf, uint64_t len);
int soil_server_get_stats(soil_server* server, soil_server_stats* out);

/* ---- instrumentation (no reference counterpart: the reference has only
 * wall-clock thermo columns, soil_print/src/lib.rs:20-26) ------------------ */
/* Kernels this library has launched in this process. */
uint64_t soil_kernel_launches(void);
/* Name of the kernel that computes the built-in consumer's forces on a
 * single system under the current SOIL_FORCE setting ("k_force_csr", ...). */
const char* soil_consumer_kernel(void);
/* Phase timers of soil_step: CUDA events recorded on the system stream
 * around each phase.  0 integrate (deform + initial, with the previous final
 * fused in), 1 zero, 2 pbc, 3 sort, 4 borders, 5 forward, 6 neighbor,
 * 7 force, 8 reverse, 9 final. */
#define SOIL_NUM_TIMERS 10
/* Time the phases whose bit is set in `mask` (0 disables); resets the sums. */
int soil_sys_set_timing(soil_sys* sys, uint32_t mask);
/* Summed milliseconds, kernel launches and timed intervals per timer. */
int soil_sys_get_timing(soil_sys* sys, double* ms, uint64_t* launches, uint64_t* intervals);
const char* soil_timer_name(int32_t i);

#ifdef __cplusplus
}
#endif
#endif /* SOIL_CUDA_H */
