/* ddg.h - C ABI of the B200 double-dummy solver (libddg.so).
 *
 * Card model (the reference's, src/dd.h:13-14): a hand is a uint64 with bit suit*16+rank,
 * suits 0..3 = S,H,D,C, ranks 0..12 = 2..A; seats 0..3 = N,E,S,W; strains 0..4 =
 * C,D,H,S,NT. A deal is 4 hands N,E,S,W (the 32-byte input record of dd_stream,
 * gpu/stream_main.cu:4-8). A result is 20 bytes, tricks[strain][declarer] (the payload of
 * the 28-byte output record, gpu/stream_main.cu:298-302); E/W declarers get 13 - NS tricks
 * also for endings with fewer than 13 cards (src/dd.h:922,937). 255 = not solved (stopped
 * by the time limit).
 *
 * Every call returns DDG_OK (0) or a negative DDG_E* code; ddg_last_error() then gives a
 * one-line message (thread-local). The reference has no error returns: its preconditions
 * (disjoint hands of equal size 1..13, strain 0..4, TT_LOG2 >= 9) are checked here.
 *
 * Threading: a ddg_solver is used by one host thread at a time. Solvers on different
 * devices are independent.
 */
#ifndef DDG_H
#define DDG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DDG_OK 0
#define DDG_E_ARG -1     /* invalid argument or deal */
#define DDG_E_CUDA -2    /* CUDA error (message names it) */
#define DDG_E_MEMORY -3  /* the TT / state pool does not fit on the device */
#define DDG_E_STATE -4   /* call out of order (e.g. stream not open) */
#define DDG_E_TIMEOUT -5 /* a bounded device wait gave up */

typedef struct ddg_solver ddg_solver;
typedef struct ddg_guide ddg_guide; /* the learned guide (below) */

/* Solver configuration. Zero fields take the defaults. Mirrors the reference's knobs:
 * TT_LOG2 (gpu/gpu_main.cu:192), THREADS (:202), PER_LEAD (gpu/stream_main.cu:167),
 * TIME_LIMIT (gpu/gpu_main.cu:247). */
typedef struct ddg_config {
  int tt_log2;          /* TT buckets per lane = 2^tt_log2, 9..20; default 10 (320 KB per lane) */
  int lanes;            /* solver lanes (GPU threads, one search each); default: fill the GPU */
  int block;            /* threads per block (lanes per block): 64, 128, 256 or 512; default 512 */
  int jobs_per_deal;    /* 5 = one job per strain, the 4 leads share a TT; 20 = one per lead */
  int device;           /* CUDA device ordinal */
  int schedule;         /* 0: block-phase kernel (all warps of a block run each stage phase
                           in turn over the block's compacted lanes); 1: queue kernel (each
                           warp takes up to 32 lanes from the fullest per-stage queue of its
                           block, no block barriers); 2: block-phase kernel with ENTER
                           inside a trick run in the cheap pass (four phases, not five) */
  int min_blocks;       /* resident blocks per SM the kernel is compiled for (register cap):
                           block 64: 1; block 128: 1, 4, 6; block 256: 1..3; block 512: 1;
                           0 = 2 for block 256, else 1 */
  double time_limit_s;  /* stop after this many seconds (unfinished results = 255); 0 = none */
  double mem_fraction;  /* largest share of free device memory the pool may take; default 0.85 */
  int help;             /* 1: once the job queue is empty, idle lanes take over untried sibling
                           moves of busy lanes in their block (same tricks, other node counts);
                           0: every job is searched by one lane, nodes equal the reference's */
  int free_below;       /* a block with fewer busy lanes than this runs free-running rounds
                           (each warp steps its own lanes, no phases): faster lanes in the
                           batch's tail. 0 = 96, -1 = never */
  int free_steps;       /* stages per lane per free-running round; 0 = 256 */
  int phase_spread;     /* block-phase kernel: 0 = a phase's lanes fill whole warps in turn;
                           1 = they go round-robin over all warps of the block */
  int cheap_limit;      /* most cheap stages (returns, next moves, job starts) a lane runs in
                           one pass of the block-phase kernel: a lane with a long chain of
                           returns no longer holds up the block's other phases; 0 = 3, -1 =
                           no limit */
  int help_share_tt;    /* with help: 0 or 1 = a helper searches its task in the donor's TT
                           (all lanes on parts of one job share what they learn; 40 hard
                           deals per lead: 129 s against 191 s without helping); -1 = in
                           its own TT (240+ s) */
  int flat_moves;       /* block-phase kernel: 0 or 1 = the lead-move phase computes the DDS
                           weights of all its (lane, candidate) pairs side by side over the
                           block's threads (13-card deals: 696 against 663 M nodes/s); -1 =
                           each lane's thread loops over its candidates; same move order and
                           node counts either way */
  int free_pack;        /* free-running rounds: the block's busy lanes are spread over
                           ceil(busy / free_pack) warps (at least enough warps to hold them,
                           at most all); 0 = one lane to a warp up to 8 busy lanes, else 32
                           to a warp (13-card deals, 68 busy lanes per block: 169 M nodes/s
                           packed against 74 M one to a warp) */
} ddg_config;

/* Counters of one solve call (device-side counters, summed over lanes). */
typedef struct ddg_stats {
  uint64_t nodes;          /* search nodes (dd_enter calls in the reference) */
  uint64_t tt_probes;      /* TT probes */
  uint64_t tt_hits;        /* probes that decided the node */
  uint64_t tt_stores;      /* TT stores that reached the bucket */
  uint64_t tt_bytes;       /* TT bytes read + written (tag lines, entries) */
  uint64_t enter_exit[7];  /* ENTER outcomes: trivial, last trick, TT hit, quick tricks,
                              later tricks, 2nd-hand quick tricks, expanded; counted by
                              libddg_check.so only (zero in libddg.so, whose per-lane
                              counters are kept small to leave shared memory to L1) */
  uint64_t phase_warps[5]; /* warp passes per phase of the block loop: cheap stages, ENTER at
                              a trick start, ENTER inside a trick, lead moves, follow moves */
  uint64_t phase_items[5]; /* lanes served by those passes; items / (32 * warps) is the
                              phase's warp efficiency */
  uint64_t phase_cycles[5]; /* SM clock cycles spent in each phase, summed over blocks */
  uint64_t free_rounds;    /* free-running rounds (blocks with few busy lanes), summed over blocks */
  uint64_t free_cycles;    /* SM clock cycles of those rounds */
  uint64_t iterations;     /* block iterations, summed over blocks */
  uint64_t tasks;          /* sibling-move tasks handed to helping lanes */
  int64_t jobs_done;       /* finished jobs */
  double kernel_ms;        /* device time of the solve kernel (CUDA events) */
  int lanes;               /* lanes launched */
  int grid, block;         /* launch shape */
  uint64_t tt_entry_reads; /* tag-matched entries read by probes (16 bytes each): the TT's
                              algorithmic bytes are 64 * probes + 16 * entry reads + 80 * stores */
} ddg_stats;

const char* ddg_version(void);
const char* ddg_last_error(void);

/* Default configuration (fills `cfg`). */
void ddg_config_default(ddg_config* cfg);

/* Creates a solver on cfg->device: allocates the per-lane TTs and search stacks once
 * (lanes * (320 << tt_log2 + 2.6 KB) bytes) and clears the TT tags. */
int ddg_solver_create(const ddg_config* cfg, ddg_solver** out);
void ddg_solver_destroy(ddg_solver* s);
/* Lanes actually allocated, and the bytes of device memory the pool holds. */
int ddg_solver_lanes(const ddg_solver* s);
int64_t ddg_solver_bytes(const ddg_solver* s);
/* Search nodes over all calls of this solver (the reference's DDCtx::nodes, src/dd.h:119). */
uint64_t ddg_solver_nodes(const ddg_solver* s);
/* Later solves write each job's completion time (device global timer, ns; 0 = not
 * finished) into d_job_end_ns[job] (device memory, n * jobs_per_deal words, job =
 * deal * jobs_per_deal + strain (jpd 5) or + strain * 4 + declarer (jpd 20)); NULL stops
 * it. No counterpart in the reference, which reports no latency (per-job tails, p99). */
int ddg_solver_set_job_times(ddg_solver* s, uint64_t* d_job_end_ns);
/* The same for the time each job was taken by a lane (its search time is end - start);
 * d_job_start_ns: n * jobs_per_deal words, 0 = not started; NULL stops it. */
int ddg_solver_set_job_starts(ddg_solver* s, uint64_t* d_job_start_ns);

/* Solves n deals (hands: n*4 uint64, host memory) for all 5 strains and 4 declarers;
 * out20: n*20 bytes, host memory. Replaces the reference's batch of dd_solve_strain calls
 * (src/dd.h:926, cpu/cpu_main.cpp:53-68, gpu/gpu_main.cu:44-48). */
int ddg_solve_batch(ddg_solver* s, const uint64_t* hands, int64_t n, uint8_t* out20, ddg_stats* st);

/* As ddg_solve_batch, each declarer's NS tricks found by stepping from a seed
 * (ns_seed20: n*20, NS tricks per [strain][declarer]); a right seed costs two searches.
 * Replaces dd_solve_strain_guess (src/dd.h:915) / dd_ns_tricks_from (src/dd.h:898). */
int ddg_solve_batch_seeded(ddg_solver* s, const uint64_t* hands, int64_t n, const int8_t* ns_seed20,
                           uint8_t* out20, ddg_stats* st);

/* Device-memory form: d_hands (n*4), d_seed20 (n*20 or NULL = binary search), d_out20
 * (n*20), d_job_nodes (n*jobs_per_deal search nodes per job, or NULL) are device
 * pointers; the solve is enqueued on `stream` (a cudaStream_t, NULL = legacy default)
 * and this call waits for it. */
int ddg_solve_device(ddg_solver* s, const uint64_t* d_hands, int64_t n, const int8_t* d_seed20,
                     uint8_t* d_out20, uint64_t* d_job_nodes, void* stream, ddg_stats* st);

/* ddg_solve_device as one CUDA graph (counter, table and task-pool clears and the
 * persistent solve kernel), instantiated on the first call and replayed while d_hands,
 * n, d_seed20 and d_out20 stay the same (a new set rebuilds it); the solver's job-time
 * buffer, when set, is part of the graph. No counterpart in the reference (its batch is a
 * plain launch, gpu/gpu_main.cu:256). */
int ddg_solve_graph(ddg_solver* s, const uint64_t* d_hands, int64_t n, const int8_t* d_seed20, uint8_t* d_out20,
                    void* stream, ddg_stats* st);

/* ddg_solve_device with the learned guide's two seams (device buffers, n*20, indexed
 * [deal][strain][declarer] like the results; NULL = unused): d_hint20 = a lead card
 * (suit*16+rank) to try first at the job's root while the TT has no move for it (-1 =
 * none; cards not in the leader's hand are ignored) - the reference's move-hint seam,
 * src/dd.h:562,594-600; d_best20 receives a best lead for each answer (the root card that
 * decided the last search going the leader's way, -1 when no lead was needed), the labels
 * of the guide's move head (src/dd.h:847). Seeds, hints and labels never change a trick. */
int ddg_solve_device_ex(ddg_solver* s, const uint64_t* d_hands, int64_t n, const int8_t* d_seed20,
                        const int8_t* d_hint20, uint8_t* d_out20, int8_t* d_best20, uint64_t* d_job_nodes,
                        void* stream, ddg_stats* st);

/* Resumable (time-sliced) solve of n deals on device buffers. ddg_solve_begin sets it up
 * (results = 255 until solved); each ddg_solve_continue runs it for at most `seconds` and
 * returns with every lane's search state kept in device memory, so the next call goes on
 * where this one stopped; *finished = 1 once every result is written. `hands_host`
 * (n*4 uint64, pinned for an asynchronous copy) is copied over d_hands before the slice
 * and `out20_host` (n*20) receives d_out20 after it, when not NULL. st = this slice's
 * counters (jobs_done = jobs finished in the slice). The reference's TIME_LIMIT
 * (gpu/gpu_main.cu:247-266) ends its kernel and drops unfinished jobs; a slice keeps them.
 * Another solve call on the same solver ends a resumable solve. */
int ddg_solve_begin(ddg_solver* s, const uint64_t* d_hands, int64_t n, const int8_t* d_seed20,
                    uint8_t* d_out20, void* stream);
int ddg_solve_continue(ddg_solver* s, double seconds, const uint64_t* hands_host, uint8_t* out20_host,
                       void* stream, ddg_stats* st, int* finished);
/* ddg_solve_begin with the guide's root leads (d_hint20, as in ddg_solve_device_ex). */
int ddg_solve_begin_ex(ddg_solver* s, const uint64_t* d_hands, int64_t n, const int8_t* d_seed20,
                       const int8_t* d_hint20, uint8_t* d_out20, void* stream);

/* Streams (continuous batching; the reference's dd_stream, gpu/stream_main.cu:38-114,
 * 189-332). A stream keeps the solver's lanes running as one persistent kernel that takes
 * jobs from a device-resident ring of deals while the host keeps publishing new ones; a
 * deal's 28-byte record (uint64 0-based submission index, then tricks[strain][declarer],
 * gpu/stream_main.cu:298-302) is available as soon as its last job ends, out of order.
 * ring_slots: power of two, 64..4M (0 = 65,536). Admission: ddg_stream_submit accepts
 * deals only while ring slots are free and at most 2 * lanes jobs are in flight (each job
 * holds a lane and its TT); *accepted says how many of the n it took, in order. Deals wait
 * for nothing but a free lane: requests that arrive while others are on the GPU start as
 * lanes free up. Lanes that find no deal for idle_timeout_s (0 = 30 s) end; the next
 * submit or poll launches the kernel again. While a stream is open the solver's other
 * calls return DDG_E_STATE. Runs on the block-phase kernel (schedule 0 or 2), helping off. */
typedef struct ddg_stream ddg_stream;
int ddg_stream_open(ddg_solver* s, int ring_slots, double idle_timeout_s, ddg_stream** out);
/* A stream whose deals are searched with the learned guide (`guide`, on the solver's
 * device): every submit runs the guide on the new deals before they are published, and
 * each job steps from the guide's NS seed with its lead tried first at the root, as
 * ddg_solve_device_ex. The guide's kernels need SMs the persistent solve kernel leaves
 * free: the solver must have at most (SMs - 2) * block lanes (else DDG_E_STATE). */
int ddg_stream_open_guided(ddg_solver* s, int ring_slots, double idle_timeout_s, ddg_guide* guide,
                           ddg_stream** out);
int ddg_stream_submit(ddg_stream* st, const uint64_t* hands, int64_t n, int64_t* accepted);
/* Copies up to `max` finished deals' 28-byte records into rec28; *got = how many. */
int ddg_stream_poll(ddg_stream* st, uint8_t* rec28, int64_t max, int64_t* got);
/* Deals submitted and not yet polled; the admission limit on them. */
int64_t ddg_stream_in_flight(const ddg_stream* st);
int64_t ddg_stream_capacity(const ddg_stream* st);
/* Ends the stream: drain = 1 waits until every submitted deal is solved, 0 stops the
 * lanes at once (deals in flight are dropped, as the reference's bench stop,
 * gpu/stream_main.cu:320-323). Records not polled are dropped. st_out = counters over the
 * stream's life (tasks = kernel launches). Frees the stream. */
int ddg_stream_close(ddg_stream* st, int drain, ddg_stats* st_out);

/* One strain of one deal, declarers N,E,S,W (tricks as ints): the reference's
 * dd_solve_strain (src/dd.h:926) and dd_solve_strain_guess (src/dd.h:915; ns4 = NS seeds,
 * NULL = binary search). One job on the GPU with a fresh TT generation, so its node count
 * is the reference's for the same call. For many deals use ddg_solve_batch. */
int ddg_solve_strain(ddg_solver* s, const uint64_t* hands4, int strain, const int* ns4, int* out4);

/* NS tricks of one lead: `leader` (0..3 = N,E,S,W) on lead in `strain`, with a fresh TT
 * generation. stepping = 0: the reference's dd_ns_tricks (src/dd.h:877-891), a binary
 * search over targets whose first target is `guess` clamped to 1..13; stepping = 1:
 * dd_ns_tricks_from (src/dd.h:898-912), stepping up or down from `guess` clamped to
 * 0..tricks left (a right guess costs two searches). The reference's calls read the deal
 * and trump from the caller's DDCtx; here they are arguments. *ns_out = NS tricks. */
int ddg_ns_tricks(ddg_solver* s, const uint64_t* hands4, int strain, int leader, int guess, int stepping,
                  int* ns_out);

/* The learned guide (no counterpart in the reference; it plugs into the reference's seams
 * for an N seed, src/dd.h:898-924, and a move hint, src/dd.h:562,594-600). An MLP of
 * 217 inputs (52 cards x 4 owners one-hot, 5 strains, 4 leaders) -> 256 GELU -> 256 GELU
 * -> 14 NS-trick classes + 52 lead-card scores, BF16 weights with FP32 accumulation, run
 * forward and backward by this library's tcgen05 tensor-core kernels. Parameters: a flat
 * fp32 array of ddg_guide_param_count() values: W1[256][256] (inputs padded to 256),
 * b1[256], W2[256][256], b2[256], W3[80][256] (outputs padded to 80), b3[80]. An example
 * is (deal, strain, declarer) = index deal*20 + strain*4 + declarer, leader = declarer+1. */
int64_t ddg_guide_param_count(void);
/* max_rows: examples per training step / inference pass, a multiple of 128. params: the
 * initial parameters (NULL = zeros). */
int ddg_guide_create(int device, int max_rows, const float* params, ddg_guide** out);
void ddg_guide_destroy(ddg_guide* g);
int ddg_guide_get_params(ddg_guide* g, float* params);
int ddg_guide_set_params(ddg_guide* g, const float* params);
/* One step on the examples rows[0..n_rows) of the deals d_hands with labels d_tricks20
 * (the solver's tables, 255 = no label) and d_best20 (best leads, -1 = none): softmax
 * cross-entropy of both heads (the lead head over the leader's cards), gradients by
 * backpropagation, then Adam with learning rate lr (lr <= 0: no update). stats3 (optional,
 * host) = mean loss, trick-head hits, labelled rows; grad_host (optional) = the gradients
 * in the parameter layout. */
int ddg_guide_train_step(ddg_guide* g, const uint64_t* d_hands, const uint8_t* d_tricks20, const int8_t* d_best20,
                         const int64_t* rows_host, int n_rows, float lr, float* stats3, float* grad_host);
/* For n deals: d_seed20 = predicted NS tricks per [strain][declarer] (seeds for
 * ddg_solve_batch_seeded / ddg_solve_device_ex) and d_hint20 = the leader's card with the
 * highest lead score (for ddg_solve_device_ex); either may be NULL. Device buffers. */
int ddg_guide_predict(ddg_guide* g, const uint64_t* d_hands, int64_t n, int8_t* d_seed20, int8_t* d_hint20);

/* No counterpart in the reference. A solve that allocates nothing, for callers that may
 * not call cudaMalloc/cudaFree: a process whose device memory is already reserved by
 * another allocator (a framework's caching pool), a latency-critical loop that cannot take
 * cudaFree's device-wide synchronisation, or code that must not fail for lack of memory at
 * run time. Its working memory is a static device array reserved when libddg.so's module
 * loads: 256 lanes with 2^9-bucket TTs, their stacks and counters (42.6 MB); no solver
 * object is needed. d_hands (n*4 uint64, 16-byte aligned) and d_out20 (n*20) are the
 * caller's device buffers, n <= 1,048,576 deals (larger n: DDG_E_ARG); one job per
 * (deal, strain), binary search, tricks equal to ddg_solve_batch's. The call only enqueues
 * two memsets and one launch on `stream` (a cudaStream_t, NULL = legacy default) and does
 * not wait. The first call on each device looks up the array's address
 * (cudaGetSymbolAddress) and must come before any stream capture on that device. Calls
 * share the array: they must not overlap (serialise them on one stream or synchronise in
 * between); overlapping calls race and their results are undefined. */
int ddg_solve_static(const uint64_t* d_hands, int64_t n, uint8_t* d_out20, void* stream);

/* Checks a deal (4 disjoint hands of equal size 1..13); DDG_OK or DDG_E_ARG. */
int ddg_check_deal(const uint64_t* hands4);

/* Seeded deal generator used by the command lines and the benchmarks: splitmix64 and a
 * Fisher-Yates shuffle of the 52 cards; deal i uses its own stream, so any range can be
 * made alone. Cards 0..4k-1 of the shuffle go round-robin to N,E,S,W (as the reference's
 * random_deals, gpu/gpu_main.cu:154-163). hands: n*4. */
void ddg_make_deals(uint64_t seed, int64_t first, int64_t n, int k, uint64_t* hands);

/* Uneven-hardness deals: K drawn uniformly from k_min..k_max cards per seat, and a share
 * `skew` of the deals skewed: one seat holds min(7..10, K) cards of one suit and another
 * seat is void in it (the rest dealt round-robin from the shuffle). No counterpart in the
 * reference (its configurations name the workload, not a generator). hands: n*4. */
void ddg_make_deals_mixed(uint64_t seed, int64_t first, int64_t n, int k_min, int k_max, double skew,
                          uint64_t* hands);

#ifdef __cplusplus
}
#endif
#endif /* DDG_H */
