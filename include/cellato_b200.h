/*
 * cellato_b200.h -- C-ABI of the B200 (sm_100a) bit-plane traverser backend
 * for Cellato.
 *
 * Plain C types only: device and host memory are `void*`, sizes are
 * `int64_t`/`size_t`, a CUDA stream is passed as `void*` (a cudaStream_t,
 * NULL = the legacy default stream, which is what the reference's traversers
 * launch on: traversers/cuda/simple.cuh:66-67).
 *
 * Every function returns CB2_OK (0) or a negative CB2_E* code; the message of
 * the last failure on the calling thread is available from cb2_last_error().
 * This replaces the reference's exception convention (CUCH -> CudaError,
 * traversers/cuda_utils.cuh:37-47; std::runtime_error / std::invalid_argument
 * for invalid configurations, traversers/cuda/temporal.hpp:57-83): the C++
 * wrapper in cellato_b200/traverser.hpp rethrows those types.
 *
 * Cells, layouts and words follow the reference exactly:
 *   - a cell's value is its state-dictionary index
 *     (memory/state_dictionary.hpp:10-42);
 *   - CB2_LAYOUT_BIT_PLANES is memory/bit_planes_grid.hpp:234-270: P planes,
 *     each y rows of x/W words, bit i of word xw = cell xw*W + i;
 *   - CB2_LAYOUT_BIT_ARRAY is memory/bit_array_grid.hpp:80-333;
 *   - CB2_LAYOUT_TILED_BIT_PLANES is memory/tiled_bit_planes_grid.hpp:35-290;
 *   - CB2_LAYOUT_STANDARD is one cell per 1 or 4 bytes, row-major
 *     (memory/standard_grid.hpp:36-60).
 * Boundaries are toroidal on all four edges (memory/interface.hpp:31-36).
 */
#ifndef CELLATO_B200_H
#define CELLATO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CB2_ABI_VERSION 4

/* ---- status codes ------------------------------------------------------- */
#define CB2_OK 0
#define CB2_EINVAL (-1)      /* invalid argument or unsupported configuration */
#define CB2_ECUDA (-2)       /* a CUDA runtime call failed                    */
#define CB2_ENOMEM (-3)      /* device memory or the memory budget exhausted  */
#define CB2_ESTATE (-4)      /* a cell value outside the state dictionary     */
#define CB2_ETIMEOUT (-5)    /* a bounded device-side wait gave up            */
#define CB2_ENOTFOUND (-6)   /* unknown request / automaton                    */

/* ---- layouts (experiments/test_suites.hpp:39-125) ------------------------ */
#define CB2_LAYOUT_STANDARD 0
#define CB2_LAYOUT_BIT_ARRAY 1
#define CB2_LAYOUT_BIT_PLANES 2
#define CB2_LAYOUT_TILED_BIT_PLANES 3

/* ---- bundled automata (src/automata/registry.hpp:17-27) ----------------- */
#define CB2_GAME_OF_LIFE 0 /* "game-of-life", P=1 (game_of_life/config.hpp)   */
#define CB2_WIRE 1         /* "wire", P=2 (wire/config.hpp)                    */
#define CB2_EXCITABLE 2    /* "excitable", P=3 (excitable/config.hpp)          */

int cb2_abi_version(void);

/* Message of the last failing call on this thread ("" if none). */
const char* cb2_last_error(void);

/* Automaton registry.  Replaces the compile-time catalog lookup by name
 * (suite::is_for, experiments/test_suites.hpp:190-195).  Returns the id or
 * CB2_ENOTFOUND. */
int cb2_automaton_lookup(const char* name);
/* name, bit-planes P and number of states of automaton `id`. */
int cb2_automaton_info(int id, const char** name, int* planes, int* states);
/* Number of registered automata; ids run from 0 to this minus one.  Ids 0-2
 * (game-of-life, wire, excitable) run hand-written networks; the others are
 * Cellato DSL automata (the bundled set, src/automata/registry.hpp:1-35, and
 * "<name>:dsl" twins of the first three) whose type-level AST
 * (core/ast.hpp) the library lowered to word-wide code at build time. */
int cb2_automaton_count(void);
/* Fingerprint of the rule registered as automaton `id`: a structural hash of
 * its Cellato config's algorithm type and state dictionary
 * (include/cellato_b200/fingerprint.hpp).  The reference instantiates each
 * suite for the config type and so always evaluates that config's own rule
 * (experiments/test_suites.hpp:189-195); the drop-in traverser compares this
 * value with its config's fingerprint so that a config whose name matches a
 * registered automaton but whose rule differs is rejected instead of run.
 * CB2_ENOTFOUND if the id is unknown or the library was built without the
 * Cellato headers. */
int cb2_automaton_fingerprint(int id, uint64_t* fingerprint);
/* State value of each dictionary index of automaton `id` (index_to_state,
 * memory/state_dictionary.hpp:10-62, as an integer): writes up to `capacity`
 * values and returns the number of states. */
int cb2_automaton_values(int id, int64_t* values, int capacity);

/* ---- tuning ------------------------------------------------------------- */
/* Knobs of one run; 0 in any field means "choose automatically" (autotuned
 * entry if one is cached for this automaton and size, else a heuristic).
 * Replaces --temporal_steps / --temporal_tile_size_y / --cuda_block_size_*
 * (experiments/run_params.hpp:10-43). */
typedef struct cb2_tuning {
    int temporal_steps;  /* generations per HBM round trip: 1, 2, 4, 8, 16,
                            32                                              */
    int tile_rows;       /* output rows per strip task (one CTA)            */
    int words_per_lane;  /* 32-bit words per lane: 1, 2 or 4                */
    int levels_per_warp; /* generations each warp of the CTA holds; the CTA
                            has temporal_steps / levels_per_warp warps      */
    int rows_per_step;   /* rows each warp passes on between two CTA
                            barriers: 1, 2 or 4                             */
} cb2_tuning;

/* ---- caller-owned device planes ----------------------------------------- */
/* Advances a grid held in caller-owned device memory, the way a reference
 * traverser's run(steps) does (traversers/cuda/simple.cuh:44-79,
 * temporal.cuh:153-245): `a` holds the input planes (P pointers, each
 * y_size * x_size/32 32-bit words, laid out as CB2_LAYOUT_BIT_PLANES), `b` is
 * the second buffer of the double buffer.  The two buffers alternate; on
 * return *result_in_b says which one holds generation `steps`.  x_size must
 * be a multiple of 32.  Launches only; nothing is synchronised. */
int cb2_run_bit_planes(int automaton, void* const* a, void* const* b, int64_t x_size, int64_t y_size, int64_t steps,
                       const cb2_tuning* tuning, void* stream, int* result_in_b);
/* The same starting at generation `time_step` (the 0-based time_step the
 * reference's evaluators read: alternate_algorithms, Margolus blocks and
 * probability draws depend on it, traversers/cpu/simple.hpp:59-62) with
 * random seed `seed` (run_params::seed, 42 in cb2_run_bit_planes). */
int cb2_run_bit_planes_at(int automaton, void* const* a, void* const* b, int64_t x_size, int64_t y_size,
                          int64_t time_step, int64_t steps, uint64_t seed, const cb2_tuning* tuning, void* stream,
                          int* result_in_b);

/* Bytes of the static device scratch behind cb2_run_bit_planes_in_place. */
#define CB2_STATIC_SCRATCH_BYTES (16u << 20)

/* Allocation-free form of cb2_run_bit_planes for callers that cannot call
 * cudaMalloc (a host application that owns all device memory and forbids
 * plugins to allocate, or a step loop that must not allocate).  It has no
 * counterpart in the reference.  `planes` (P consecutive planes in one
 * allocation, CB2_LAYOUT_BIT_PLANES) hold generation `time_step` and, in
 * stream order, receive generation time_step + steps.  `time_step` and `seed`
 * mean what they mean in cb2_run_bit_planes_at: rules that read the
 * generation or the seed (alternate_algorithms, Margolus blocks, probability
 * draws) need them, so a step loop of N calls passes its running generation
 * count and one seed, and then matches one run of N*steps generations.
 * The second buffer of the double buffer is a
 * file-scope __device__ array of CB2_STATIC_SCRATCH_BYTES that every GPU
 * loading this library holds until exit; grids whose planes are larger are
 * rejected with CB2_EINVAL.  No cudaMalloc / cudaFree or allocating routine
 * is called.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  All calls on a device share the array, so
 * calls that overlap on the GPU (different streams, or different host
 * threads) race; serialise them. */
int cb2_run_bit_planes_in_place(int automaton, void* const* planes, int64_t x_size, int64_t y_size,
                                int64_t time_step, int64_t steps, uint64_t seed, const cb2_tuning* tuning,
                                void* stream);

/* ---- owning device grids -------------------------------------------------- */
/* A device-resident grid: P bit-planes, double-buffered, generation counter.
 * Mirrors grid::to_cuda / to_cpu / free_cuda_memory of the reference layouts
 * (memory/bit_planes_grid.hpp:146-190) plus traverser::init / run /
 * fetch_result (traversers/cuda/simple.hpp:25-104). */
typedef struct cb2_grid cb2_grid;

/* x_size must be a multiple of 32 (the 32-bit word of the device layout). */
int cb2_grid_create(int automaton, int64_t x_size, int64_t y_size, cb2_grid** out);
int cb2_grid_destroy(cb2_grid* grid);

/* Host image <-> device planes.  `host` may be pageable or pinned memory;
 * `bytes` must equal cb2_layout_bytes(...).  word_bits: 32 or 64 for the
 * packed layouts, 8 or 32 (bytes per cell x 8) for CB2_LAYOUT_STANDARD.
 * Upload returns CB2_ESTATE if a standard-layout cell is not a dictionary
 * index.  Both calls complete the copy before returning. */
int cb2_grid_upload(cb2_grid* grid, int layout, int word_bits, const void* host, size_t bytes, void* stream);
int cb2_grid_download(cb2_grid* grid, int layout, int word_bits, void* host, size_t bytes, void* stream);
/* The same copies enqueued on `stream` without waiting for them, so that a
 * caller streaming a sequence of grids can overlap one grid's upload and
 * another's download with a third's run (two copy streams and events).  No
 * counterpart in the reference, whose traversers copy synchronously in init
 * and fetch_result.  The host image must stay valid and unchanged (upload)
 * or unread (download) until the stream has passed the copy; from pinned
 * host memory the copy runs beside kernels.  A grid's upload, runs and
 * download must still be ordered (one stream, or events).  The standard
 * layout is refused by the upload (its cells are checked on the host:
 * cb2_grid_upload). */
int cb2_grid_upload_async(cb2_grid* grid, int layout, int word_bits, const void* host, size_t bytes, void* stream);
int cb2_grid_download_async(cb2_grid* grid, int layout, int word_bits, void* host, size_t bytes, void* stream);
/* Size of a layout's host image for a grid of this automaton and size. */
int64_t cb2_layout_bytes(int automaton, int layout, int word_bits, int64_t x_size, int64_t y_size);

/* Seeded input on the device: cell i = y*x_size + x draws
 * u = SplitMix64(seed + (i+1)*0x9E3779B97F4A7C15) >> 11 and takes state
 * index #{j : thresholds[j] <= u}; thresholds are cumulative probabilities
 * times 2^53 (fewer than the automaton's states, at most 31). */
int cb2_grid_fill_random(cb2_grid* grid, uint64_t seed, const uint64_t* thresholds, int n_thresholds, void* stream);

/* Advances the grid `steps` generations (asynchronous on `stream`); the
 * first is generation cb2_grid_time_step(grid), drawn with the grid's seed. */
int cb2_grid_run(cb2_grid* grid, int64_t steps, const cb2_tuning* tuning, void* stream);
/* Random seed of stochastic rules (default 42, run_params::seed). */
int cb2_grid_set_seed(cb2_grid* grid, uint64_t seed);
/* Sets the generation counter (the time_step of the next generation). */
int cb2_grid_set_time_step(cb2_grid* grid, int64_t time_step);

/* 16-number checksum of the current generation
 * (memory/standard_grid.hpp:182-218).  state_values maps dictionary index ->
 * state value (NULL = the automaton's own, cb2_automaton_values).
 * Synchronises `stream`. */
int cb2_grid_checksum(cb2_grid* grid, const int64_t* state_values, int n_values, uint64_t out[16], void* stream);

/* Device pointers of the current generation's planes (like grid::data()). */
int cb2_grid_planes(cb2_grid* grid, void** planes, int* n_planes, int64_t* words_per_plane);
/* Generations advanced since the last upload / fill. */
int64_t cb2_grid_time_step(const cb2_grid* grid);

/* ---- row bands: one grid split across GPUs -------------------------------- */
/* A rank holds its band of rows plus `ghost` rows above and below in
 * caller-owned planes (rows_total = band rows + 2 * ghost, P consecutive
 * planes).  Before each pass the caller refreshes the ghost rows next to the
 * band from the neighbouring ranks (a halo exchange of contiguous rows, e.g.
 * NCCL send/recv); the pass then advances exactly `temporal_steps`
 * generations of rows [row_first, row_first + rows_out) from in to out,
 * reading up to temporal_steps rows outside them.  The reference runs one
 * grid on one GPU (traversers/cuda/temporal.cuh:153-245); this is the
 * multi-GPU split of that run. */
int cb2_band_pass(int automaton, void* const* in, void* const* out, int64_t x_size, int64_t rows_total,
                  int64_t row_first, int64_t rows_out, int temporal_steps, const cb2_tuning* tuning, void* stream);
/* cb2_band_pass at generation `time_step` with random seed `seed`, for a
 * band whose planes' row 0 is global row `global_row0` (mod global_rows, so a
 * rank-0 band with ghost rows passes -ghost) of a grid `global_rows` tall.
 * Lowered DSL automata need these (Margolus blocks and probability draws read
 * the generation and the global row); cb2_band_pass refuses them. */
int cb2_band_pass_at(int automaton, void* const* in, void* const* out, int64_t x_size, int64_t rows_total,
                     int64_t row_first, int64_t rows_out, int temporal_steps, int64_t time_step, uint64_t seed,
                     int64_t global_row0, int64_t global_rows, const cb2_tuning* tuning, void* stream);
/* Depths of the passes a band run of `steps` generations takes: passes of
 * min(temporal_steps, ghost) generations, then the binary digits of the
 * remainder from the largest down (45 steps at depth 32: 32, 8, 4, 1).
 * Writes up to `capacity` depths and returns the number of passes (which may
 * exceed capacity), or CB2_EINVAL.  Host only: needs no GPU. */
int64_t cb2_band_schedule(int64_t steps, int temporal_steps, int ghost, int* depths, int64_t capacity);
/* Fills this rank's ghost rows for the next pass: the `k` rows above its
 * band (planes rows ghost-k .. ghost-1) from the last k band rows of the rank
 * above, the k rows below (rows ghost+band .. ghost+band+k-1) from the first
 * k band rows of the rank below, in buffer `buffer` (0: a, 1: b) of
 * cb2_band_run, enqueued on `stream` (NCCL send/recv, peer copies, or plain
 * copies for a single rank).  Returns 0, or a nonzero code that stops the run. */
typedef int (*cb2_halo_exchange_fn)(void* user, int buffer, int k, void* stream);
/* A whole band run for C and C++ hosts: `steps` generations from
 * `time_step`, in passes of cb2_band_schedule's depths, alternating between
 * the caller's buffers a and b (band_rows + 2 * ghost rows each, the band's
 * first row being global row `global_row0` of `global_rows`).  Each pass
 * overlaps the halo exchange with the band's interior: once the previous
 * pass is done, `exchange` is enqueued on `exchange_stream` while the rows
 * that need no ghost row (all but k at each edge) advance on `stream`; the
 * two k-row edges follow once the exchange has landed.  Bands thinner than
 * 3k rows run whole after the exchange.  Launches only; *result_in_b says
 * which buffer holds the result.  The reference runs one grid on one GPU
 * (traversers/cuda/temporal.cuh:153-245); this is its multi-GPU split. */
int cb2_band_run(int automaton, void* const* a, void* const* b, int64_t x_size, int64_t band_rows, int ghost,
                 int64_t time_step, int64_t steps, uint64_t seed, int64_t global_row0, int64_t global_rows,
                 const cb2_tuning* tuning, cb2_halo_exchange_fn exchange, void* user, void* stream,
                 void* exchange_stream, int* result_in_b);
/* Seeded input (cb2_grid_fill_random's stream) for caller-owned planes whose
 * row y is global row (global_row0 + y) mod global_rows of the global grid. */
int cb2_fill_random_planes(int automaton, void* const* planes, int64_t x_size, int64_t rows, int64_t global_row0,
                           int64_t global_rows, uint64_t seed, const uint64_t* thresholds, int n_thresholds,
                           void* stream);
/* The 16 tile sums (memory/standard_grid.hpp:182-218) contributed by rows
 * [row_first, row_first + row_count) of the planes, which are global rows
 * global_row0.. of a grid global_rows tall; summing the results of all
 * bands gives the global checksum.  Synchronises `stream`. */
int cb2_checksum_planes(int automaton, const void* const* planes, int64_t x_size, int64_t rows, int64_t row_first,
                        int64_t row_count, int64_t global_row0, int64_t global_rows, const int64_t* values,
                        int n_values, uint64_t out[16], void* stream);

/* ---- batches: many grids in one persistent kernel ------------------------ */
/* A batch advances each of its grids by that grid's own number of
 * generations in one persistent kernel over a queue of strip tasks, replayed
 * as a captured CUDA graph.  There is no counterpart in the reference, whose
 * traversers run one grid per launch sequence (traversers/cuda/simple.cuh:44-79);
 * cb2_batch_run_per_grid is that one-launch-per-grid path over the same grids
 * for comparison.  The grids stay owned by the caller; while they belong to a
 * batch, advance them through the batch (a grid advanced, re-uploaded,
 * re-timed or re-seeded outside it makes the next cb2_batch_run rebuild the
 * schedule).  Every registered automaton batches; a batch holding a lowered
 * DSL automaton runs a kernel over all of them, in which each grid's draws,
 * Margolus blocks and alternating algorithms follow its own generation and
 * seed (cb2_grid_set_seed, cb2_grid_set_time_step). */
typedef struct cb2_batch cb2_batch;

typedef struct cb2_batch_opts {
    int temporal_steps;   /* K of full chunks: 1, 2, 4, 8, 16 or 32 (0 = 32; batches
                             holding a lowered DSL automaton run chunks of at most 8) */
    int tile_rows;        /* output rows per strip task (0 = 768 for the hand-written
                             networks, 64 for lowered DSL rules)                       */
    long long spin_limit; /* iterations a task waits for its grid's previous chunk
                             before the run fails with CB2_ETIMEOUT (0 = ~4 s)         */
    int stall_task;       /* test hook: index of a task whose dependency is never
                             satisfied, to exercise the timeout path (-1 = none)      */
} cb2_batch_opts;

int cb2_batch_create(cb2_grid* const* grids, const int64_t* steps, int n, const cb2_batch_opts* opts,
                     cb2_batch** out);
int cb2_batch_destroy(cb2_batch* batch);
/* One pass: every grid advances its steps (asynchronous on `stream`). */
int cb2_batch_run(cb2_batch* batch, void* stream);
/* Waits for `stream`; CB2_ETIMEOUT if a task's bounded wait ran out. */
int cb2_batch_wait(cb2_batch* batch, void* stream);
/* The same work as cb2_batch_run, one launch sequence per grid. */
int cb2_batch_run_per_grid(cb2_batch* batch, void* stream);
/* Tasks per run, cell-updates per run, persistent CTAs of the kernel. */
int cb2_batch_info(const cb2_batch* batch, int64_t* tasks, double* cell_updates, int* persistent_ctas);

/* ---- serving: continuous batching of simulation requests ---------------- */
/* A server thread admits requests in arrival order while their state fits a
 * device-memory budget, keeps it resident, and advances every admitted
 * request by up to chunk_steps generations per round in one persistent batch
 * kernel; two rounds are in flight at a time, and requests that arrive
 * meanwhile join at the next round.  No
 * counterpart in the reference (one process runs one experiment,
 * experiments/experiment_manager.hpp:43-57).  per_request = 1 runs the plain
 * path instead: one request at a time, each as one launch sequence. */
typedef struct cb2_server cb2_server;

typedef struct cb2_server_opts {
    size_t memory_budget;    /* bytes of request state held at once (0 = min(150 GiB, 80% free)) */
    int max_active;          /* requests admitted at once (0 = 4096)                    */
    int chunk_steps;         /* most generations per request per round (0 = 128)       */
    int temporal_steps;      /* K of the batch kernel: 1, 2, 4, 8, 16 or 32 (0 = 32;
                                rounds holding a lowered DSL request use at most 8)  */
    int tile_rows;           /* output rows per strip task (0 = 256 for the hand-written
                                networks, 64 for lowered DSL rules)                    */
    int per_request;         /* 1 = plain one-request-at-a-time path                   */
    int task_capacity;       /* strip tasks per round (0 = 2^20)                        */
    long long spin_limit;    /* bounded wait of a task (0 = ~4 s)                       */
    long long fail_alloc_at; /* test hook: the n-th state allocation fails (0 = never)  */
    double round_cells;      /* if > 0: cell-updates a round aims at, shared by its
                                requests (0 = every request takes chunk_steps)        */
    long long direct_cells;  /* requests of at least this many cells advance through the
                                single-grid strip kernels (cb2_grid_run's plan) on a
                                second stream in each round, beside the batch kernel
                                (0 = 2^28, e.g. 16384 x 16384; negative = never)       */
} cb2_server_opts;

typedef struct cb2_request {
    int automaton;
    int64_t x_size, y_size; /* x_size a multiple of 32                                  */
    int64_t steps;
    uint64_t seed;          /* seeded input (cb2_grid_fill_random) when host_cells is NULL */
    int n_thresholds;
    uint64_t thresholds[31]; /* at most states - 1 (31: every state of a 32-state dictionary) */
    const uint8_t* host_cells; /* optional input, one dictionary index per cell; read at
                                  admission, so it must stay valid until then            */
    uint8_t* host_result;      /* optional output, one index per cell, written at completion */
} cb2_request;

#define CB2_REQ_QUEUED 0
#define CB2_REQ_ACTIVE 1
#define CB2_REQ_DONE 2
#define CB2_REQ_FAILED 3

typedef struct cb2_request_status {
    int state;          /* CB2_REQ_*                                   */
    int error;          /* status code of a failed request             */
    int64_t steps_done;
    double submit_s, admit_s, done_s; /* seconds since cb2_server_create */
    uint64_t checksum[16];            /* of the final generation        */
} cb2_request_status;

typedef struct cb2_server_stats {
    int64_t submitted, completed, failed, rounds;
    double cell_updates;
    int64_t used_bytes, budget_bytes;
    double now_s;
    double plan_s;     /* server-thread seconds spent planning and queueing rounds   */
    double wait_s;     /* server-thread seconds blocked on the GPU                   */
    int64_t tasks;     /* batch-kernel tasks run so far                              */
} cb2_server_stats;

int cb2_server_create(const cb2_server_opts* opts, cb2_server** out);
/* Thread-safe.  CB2_ENOMEM if the request alone exceeds the budget. */
int cb2_server_submit(cb2_server* server, const cb2_request* request, int64_t* id);
int cb2_server_status(cb2_server* server, int64_t id, cb2_request_status* status);
/* Blocks until the request finished (its status code) or CB2_ETIMEOUT. */
int cb2_server_wait(cb2_server* server, int64_t id, double timeout_s);
/* Blocks until every submitted request finished, or CB2_ETIMEOUT. */
int cb2_server_drain(cb2_server* server, double timeout_s);
int cb2_server_get_stats(cb2_server* server, cb2_server_stats* stats);
/* Stops the loop; requests not finished are failed. */
int cb2_server_destroy(cb2_server* server);

/* ---- tuning and measurement --------------------------------------------- */
/* Times the candidate plans for this automaton and size on the current
 * device, stores the fastest in the in-process tuning table (used whenever a
 * cb2_tuning field is 0) and returns it in *best.  `budget_ms` bounds the
 * time spent (<= 0: a default). */
int cb2_autotune(int automaton, int64_t x_size, int64_t y_size, double budget_ms, cb2_tuning* best);
/* Loads / saves the tuning table as text lines "automaton x_size y_size
 * temporal_steps tile_rows words_per_lane levels_per_warp rows_per_step"
 * (lines without the last field load with rows_per_step 1). */
int cb2_tuning_load(const char* path);
int cb2_tuning_save(const char* path);
/* The plan cb2_grid_run would use for a chunk of `steps` generations. */
int cb2_plan(int automaton, int64_t x_size, int64_t y_size, const cb2_tuning* tuning, cb2_tuning* plan);
/* The strip kernels instantiated for `automaton`: writes up to `capacity`
 * of them to out[] (temporal_steps, words_per_lane, levels_per_warp,
 * rows_per_step set; tile_rows 0) and returns how many there are.  The
 * reference's temporal traverser has one kernel shape; the table is what
 * cb2_autotune chooses from. */
int cb2_variants(int automaton, cb2_tuning* out, int capacity);

/* Measured peak of 32-bit three-input logic ops on the current device
 * (ops/s), the integer roof of the rule networks. */
int cb2_measure_lop3_peak(double* ops_per_second);

/* Logic, shift and shuffle instructions the strip kernel issues per 32-bit
 * word per generation for this automaton (the integer cost of the network),
 * for plans of two or more rows per step; with one row per step, whose rows
 * are not evaluated in pairs, game-of-life issues one logic op more and wire
 * two. */
int cb2_network_ops(int automaton, double* alu_ops_per_word, double* shuffles_per_word);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* CELLATO_B200_H */
