/*
 * gfcuda.h -- C ABI of the B200 modular-squaring engine (libgfcuda.so).
 *
 * The engine squares numbers modulo b^(2^n) + 1 on an NVIDIA B200
 * (sm_100a).  It is the drop-in backend for genefer's `transform` interface
 * (reference: src/transform.h:42-256): each single-test entry point below
 * replaces one member of that interface, cited beside it.  A genefer-side
 * `transformCUDA` class (include/transformCUDA.h) forwards to these calls.
 *
 * Conventions
 *   - Every function returns GFC_OK (0) or a negative GFC_ERR_* code and never
 *     throws; gfc_last_error() gives a message for the calling thread.
 *   - Registers hold N = 2^n signed digits in natural order (digit i has
 *     weight b^i), like the int32 vector of genefer's `gint`
 *     (src/gint.h:17-38).  Digits at rest satisfy |d| <= b/2 + 1; they are
 *     congruent, not equal, to the reference transform's digits, and
 *     gint::unbalance maps both to the same canonical residue.
 *   - Work is enqueued on the handle's CUDA stream (the one passed at
 *     creation, or a private one).  Calls that move digits to host memory
 *     synchronise that stream; the others return after enqueueing.
 *   - A gfc_transform is a batch of one test; the gfc_batch_* calls run many
 *     tests of the same n in each launch (a throughput extension with no
 *     counterpart in the reference interface).
 */
#ifndef GFCUDA_H
#define GFCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GFC_OK 0
#define GFC_ERR_ARG (-1)      /* invalid argument (size, register index, b, n) */
#define GFC_ERR_CUDA (-2)     /* CUDA runtime failure (device, memory, launch) */
#define GFC_ERR_RANGE (-3)    /* (b, n) outside the exact range of the prime sets */
#define GFC_ERR_NUMERIC (-4)  /* a device-side carry could not be absorbed */
#define GFC_ERR_STATE (-5)    /* call not valid in the current state */

typedef struct gfc_batch gfc_batch;
typedef struct gfc_batch gfc_transform;
typedef struct gfc_graph gfc_graph;

/* Message of the last failing call on this thread. */
const char *gfc_last_error(void);

/* Library version as major*10000 + minor*100 + patch. */
int gfc_version(void);

/* ------------------------------------------------------------------ single test
 * Replaces transform::create_gpu / create_ocl (src/transform.h:114-120,
 * src/transform_ocl.cpp:20-51) and the transformGPUs constructor
 * (src/transformGPU.h:945-1083).  b: base, 2 <= b < 2^31; n: 10 <= n <= 23;
 * num_regs: registers (3 for quick tests, src/genefer.h:1384); device: CUDA
 * ordinal; stream: cudaStream_t to use, or NULL for a private stream. */
int gfc_create(uint32_t b, uint32_t n, size_t num_regs, int device, void *stream, gfc_transform **out);

/* Releases all device memory (transformGPUs destructor, src/transformGPU.h:1085-1093). */
void gfc_destroy(gfc_transform *t);

/* r_0 = a  (transform::set, src/transform.h:58).  Requires a <= b/2. */
int gfc_set(gfc_transform *t, uint32_t a);

/* r_0 = r_0^2, or 2 r_0^2 when dup != 0  (transform::squareDup, src/transform.h:59). */
int gfc_square_dup(gfc_transform *t, int dup);

/* r_0 = a r_0^2 for any int32 a  (transform::squareMul, src/transform.h:60;
 * CPU reference src/transformCPUi32.h:870-874, 774-797). */
int gfc_square_mul(gfc_transform *t, int32_t a);

/* r_m = transform(r_src)  (transform::initMultiplicand, src/transform.h:61). */
int gfc_init_multiplicand(gfc_transform *t, size_t src);

/* r_0 = r_0 * r_m  (transform::mul, src/transform.h:62). */
int gfc_mul(gfc_transform *t);

/* r_dst = r_src  (transform::copy, src/transform.h:64). */
int gfc_copy(gfc_transform *t, size_t dst, size_t src);

/* Reads r_0 as N signed digits into host memory; synchronises
 * (transform::getZi via getInt, src/transform.h:54, :234-239). */
int gfc_get_zi(gfc_transform *t, int32_t *zi);

/* Writes r_0 from N host digits with |d| <= b/2, e.g. after gint::balance
 * (transform::setZi via setInt, src/transform.h:55, :241-246). */
int gfc_set_zi(gfc_transform *t, const int32_t *zi);

/* Device bytes held by the handle (transform::getMemSize, src/transform.h:66). */
size_t gfc_get_mem_size(const gfc_transform *t);

/* Bytes of state touched per squaring (transform::getCacheSize, src/transform.h:67). */
size_t gfc_get_cache_size(const gfc_transform *t);

/* Context payload (transform::saveContext / readContext, src/transform.h:69-70,
 * src/transformGPU.h:1127-1150): a tag word (GFC_CONTEXT_KIND) followed by
 * num_regs registers of N int32 digits.  gfc_context_size gives the byte size;
 * gfc_save_context synchronises; gfc_read_context returns GFC_ERR_STATE when
 * the tag or size does not match (readContext returning false). */
#define GFC_CONTEXT_KIND 0x47464342 /* "GFCB" */
size_t gfc_context_size(const gfc_transform *t, size_t num_regs);
int gfc_save_context(gfc_transform *t, void *buf, size_t size, size_t num_regs);
int gfc_read_context(gfc_transform *t, const void *buf, size_t size, size_t num_regs);

/* Number of RNS primes chosen for (b, n): 2 or 3, or 4 with packed digits
 * (two digits per coefficient of a half-length transform; the default from
 * n = 21 for a single test whose b is in the packed range); the analogue of
 * the transform kind
 * NTT2/NTT3 (src/transform.h:45, src/transform_ocl.cpp:35-50). */
int gfc_width(const gfc_transform *t);

/* Waits for all enqueued work; returns GFC_ERR_NUMERIC if a device-side check
 * failed since the last call. */
int gfc_sync(gfc_transform *t);

/* ------------------------------------------------------------------ batches of tests */

/* count (1 <= count <= 65535) tests of the same n with bases b[0..count-1] (each test picks its own
 * RNS width), num_regs registers each. */
int gfc_batch_create(const uint32_t *b, size_t count, uint32_t n, size_t num_regs, int device, void *stream,
					 gfc_batch **out);
void gfc_batch_destroy(gfc_batch *bt);
size_t gfc_batch_count(const gfc_batch *bt);

/* Per-test r_0 = a, r_dst = r_src, for all tests. */
int gfc_batch_set(gfc_batch *bt, uint32_t a);
int gfc_batch_copy(gfc_batch *bt, size_t dst, size_t src);

/* count squarings of r_0 for every test with a fixed dup flag. */
int gfc_batch_square(gfc_batch *bt, int dup, uint32_t count);

/* Uploads test `test`'s exponent (nbits bits, little-endian 32-bit words)
 * and sets its bit position to nbits - 1. */
int gfc_batch_set_exponent(gfc_batch *bt, size_t test, const uint32_t *words, uint64_t nbits);

/* Gives slot `test` a new base b (its prime set and carry constants follow);
 * the slot's registers keep their contents until overwritten.  Synchronises.
 * Used to admit a new test into a running batch.  No counterpart in the
 * reference, which runs one test per transform.  With the single-CTA plan
 * (n <= 14) a graph captured before a change of prime set is refused by
 * gfc_graph_launch (GFC_ERR_STATE); four-step graphs stay valid. */
int gfc_batch_assign(gfc_batch *bt, size_t test, uint32_t b);

/* Reserved slots (no counterpart in the reference, which runs one test per
 * transform; used by the serving loop, gfc_server_*).  gfc_batch_reserve
 * allocates, once, room for an exponent of up to max_bits bits in every slot
 * and pinned host staging; afterwards gfc_batch_admit and gfc_batch_set_exponent
 * (for nbits <= max_bits) allocate nothing and do not synchronise: they
 * enqueue their copies on the batch stream and return. */
int gfc_batch_reserve(gfc_batch *bt, uint64_t max_bits);

/* Admits a new test into slot `test` of a reserved batch: base b (its prime
 * set and carry constants), r_0 = r_1 = 1 (genefer's start, src/genefer.h:492-497),
 * exponent words (nbits <= max_bits) and bit position nbits - 1, as one
 * asynchronous sequence on the batch stream.  `words` may be reused when the
 * call returns.  A change of prime set under the single-CTA plan makes graphs
 * captured before it refuse to launch (GFC_ERR_STATE), as gfc_batch_assign. */
int gfc_batch_admit(gfc_batch *bt, size_t test, uint32_t b, const uint32_t *words, uint64_t nbits);

/* Register `reg` of one test to / from host memory, enqueued on the batch
 * stream without waiting: the host buffer (pinned for a truly asynchronous
 * copy) must stay valid until the stream has passed the copy. */
int gfc_batch_get_async(gfc_batch *bt, size_t test, size_t reg, int32_t *out);
int gfc_batch_set_async(gfc_batch *bt, size_t test, size_t reg, const int32_t *in);

/* Plan codes the engine accepts at size n (see gfc_batch_set_plan), in the
 * order gfc_batch_tune measures them; *count receives their number (up to
 * `cap` are written). */
int gfc_plan_candidates(uint32_t n, int32_t *plans, size_t cap, size_t *count);

/* Autotuner (no counterpart in the reference's OpenCL path, which picks its
 * kernel split by its own timing loop, src/transformGPU.h:841-900): for every
 * candidate plan the batch can take, `squarings` squarings of register 0 are
 * captured in a CUDA graph and replayed `replays` times between CUDA events;
 * the plan with the least device time per squaring is set (ties: the lower
 * code) and register 0 is cleared.  plans[i], us[i] (microseconds per batch
 * squaring) for i < min(cap, *count); *best the chosen plan.  Squares register 0
 * in place: tune a batch before loading its tests. */
int gfc_batch_tune(gfc_batch *bt, uint32_t squarings, uint32_t replays, int32_t *plans, float *us, size_t cap,
				   size_t *count, int32_t *best);

/* Sets every test's bit position (pos[i] < 0: the test has finished). */
int gfc_batch_set_pos(gfc_batch *bt, const int64_t *pos);
int gfc_batch_get_pos(gfc_batch *bt, int64_t *pos);

/* count squarings per test, squaring i using dup = bit (pos - i) of the
 * test's exponent, then pos -= count; tests whose position goes below zero
 * stop (the loop body of genefer::prp, src/genefer.h:508-527). */
int gfc_batch_square_exp(gfc_batch *bt, uint32_t count);

/* r_m = transform(r_src) and r_dst = r_0 * r_m, for all tests. */
int gfc_batch_init_multiplicand(gfc_batch *bt, size_t src);
int gfc_batch_mul(gfc_batch *bt, size_t dst);

/* Gerbicz-Li update d(t) <- d(t) * r for all tests: r_1 = r_0 * r_1 with r_0
 * unchanged; the same result as copy(2,0); mul(1); copy(1,0); copy(0,2)
 * (src/genefer.h:529-535) without the copies. */
int gfc_batch_gl_step(gfc_batch *bt);

/* Digits of register `reg` of one test, or of all tests (count x N). */
int gfc_batch_get_zi(gfc_batch *bt, size_t test, size_t reg, int32_t *out);
int gfc_batch_set_zi(gfc_batch *bt, size_t test, size_t reg, const int32_t *in);
int gfc_batch_get_all(gfc_batch *bt, size_t reg, int32_t *out);
int gfc_batch_set_all(gfc_batch *bt, size_t reg, const int32_t *in);

/* Kernel plan.  lr = 0: one CTA per test with the state in shared memory
 * (n <= 14); lr = 1: squarings by one thread-block cluster per test with the
 * state in the cluster's shared memory (12 <= n <= 17: eight CTAs with rows of
 * 2^9 at n = 12, sixteen with rows of 2^(n-4) at n = 13, 14, 2^(n-13) CTAs with
 * rows of 2^13 above; products use the default plan of n); 3 <= lr <= 10: four-step with R = 2^lr rows
 * (8 <= n - lr <= 13); lr = 100 + lr2 (3 <= lr2 <= 7): six-step, the column
 * transform split into 2^4 and 2^lr2 points (8 <= n - 4 - lr2 <= 13);
 * lr = 200 + l (l = 3, 4): packed digits, two base-b digits per coefficient
 * of a transform of N/2 points over four primes (8 <= n - 1 - l <= 13; every
 * base of the batch in the exact range, 2^20 <= b and (N/2)((b/2+1)(b+1))^2
 * below half the primes' product, else GFC_ERR_RANGE; gfc_batch_widths then
 * reports 4); lr = 300 + lr2: packed digits with the six-step split of the
 * half-length transform (8 <= n - 5 - lr2 <= 13).  A new batch from n = 16
 * uses packed digits when every base is in the packed range (203 at n = 16,
 * 204 at n = 17, 18, 303 at n = 19, 20, 305 at n = 21, 22, 306 at n = 23);
 * otherwise single-CTA up to n = 14,
 * four-step at n = 15, 16 (lr = n - 12), six-step above (103 at n = 17, 18,
 * 104 at n = 19, 20, 105 at n = 21, 106 at n = 22, 107 at n = 23; a lone test at
 * n = 19 too, packed or not, and at n = 12..14 the cluster plan): the fastest plans measured
 * on one B200.
 * gfc_batch_plan reads the current plan. */
int gfc_batch_set_plan(gfc_batch *bt, int lr);
int gfc_batch_plan(const gfc_batch *bt);

/* Per-test RNS width (2 or 3), into w[0..count-1]. */
int gfc_batch_widths(const gfc_batch *bt, int32_t *w);

/* Waits for all enqueued work (see gfc_sync). */
int gfc_batch_sync(gfc_batch *bt);

/* CUDA stream of the batch (cudaStream_t). */
void *gfc_batch_stream(gfc_batch *bt);

/* CUDA graphs: calls between capture_begin and capture_end are recorded (not
 * run) and replayed by gfc_graph_launch on the batch's stream. */
int gfc_batch_capture_begin(gfc_batch *bt);
int gfc_batch_capture_end(gfc_batch *bt, gfc_graph **out);
int gfc_graph_launch(gfc_graph *g);
void gfc_graph_destroy(gfc_graph *g);

/* Kernel launches issued by this process so far (all handles; a graph replay
 * counts the kernels it contains). */
uint64_t gfc_launch_count(void);

/* Kernel timing (no counterpart in the reference): runs `reps` squarings of
 * all tests (dup = 0) with a CUDA event recorded on the batch's stream around
 * every kernel, and returns the mean duration of each kernel kind in ms:
 * ms[0] single-CTA kernel (plan 0), ms[1] column-forward, ms[2] row,
 * ms[3] column-inverse + carry, ms[4] carry fix-up (0 when unused). */
int gfc_batch_time_kernels(gfc_batch *bt, uint32_t reps, float *ms);

/* Integer-pipe probe (no counterpart in the reference): Montgomery products
 * and radix-2 butterflies per second on `device`, out[0..3] = product with
 * the 32-bit primes, product with the 31-bit primes, butterfly 32-bit
 * (Montgomery root product), butterfly 31-bit (Shoup root product, as the
 * transforms of the 31-bit prime sets run it).  The roofline denominator for
 * the squaring kernels. */
int gfc_probe_int_throughput(int device, double *out);

/* ------------------------------------------------------------------ squaring without allocation
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory at the point they square (code inside another runtime's memory pool
 * or allocator lock, processes with a device-memory budget fixed at start-up,
 * hosts that forbid allocation after initialisation): count squarings (dup
 * as in gfc_square_dup) of the N = 2^n digits at device address `in`, result
 * at device address `out` (equal to `in`, or a disjoint range: a partial
 * overlap returns GFC_ERR_ARG), on `stream` (NULL: the default stream) of
 * `device`.  The input digits must satisfy |d| <= b/2 + 1.
 *  - All scratch (root tables, transform planes, carries) lives in one
 *    static device array of 5.01 MB that every GPU loading the library holds
 *    until the process exits; the call makes no cudaMalloc/cudaFree and no
 *    allocating library call.  Hence 12 <= n <= 16; larger n returns
 *    GFC_ERR_ARG.
 *  - The first call on a device resolves the array's device address and
 *    builds its root tables (again whenever n changes); make that first call
 *    before any stream capture.  The library remembers per device that the
 *    tables are built; a cudaDeviceReset discards the array's contents
 *    without the library seeing it, so after resetting a device a process
 *    must not call this entry point on that device again.
 *  - Every call shares the array: calls that overlap on the GPU (other
 *    streams, other host threads without ordering) race.  The call waits for
 *    `stream` before returning and reports a device-side carry failure as
 *    GFC_ERR_NUMERIC. */
int gfc_square_noalloc(const int32_t *in, int32_t *out, uint32_t b, uint32_t n, int dup, uint32_t count, int device,
					   void *stream);

/* ------------------------------------------------------------------ serving
 * No counterpart in the reference, which runs one test per process
 * (src/genefer.h:1360-1480).  A continuous-batching request loop on one
 * device, run by a native dispatcher thread: tests of one size n share a pool
 * of slots (one batch, its block of genefer's prp loop as one CUDA graph:
 * the Gerbicz-Li update d <- d x, src/genefer.h:529-535, then `block`
 * squarings with each slot's own exponent bits).  Between two blocks of a
 * pool, finished tests are read back and waiting tests of that size are
 * admitted into free slots (gfc_batch_admit: no allocation, no
 * synchronisation), so the pools' blocks keep overlapping on the device.
 * Pools open while the device-memory budget allows and close when idle.
 * Finished tests get genefer's Gerbicz-Li check (src/genefer.h:557-615),
 * validate_group of one size at once, on a checker batch of their own.
 * Every test reads only its own slot, base and exponent bits, so its residue
 * is the same alone and among others. */
typedef struct gfc_server gfc_server;

typedef struct gfc_server_config
{
	uint32_t block;           /* Gerbicz-Li block length B (squarings per block) */
	uint32_t validate_group;  /* finished tests checked together (0: no check) */
	uint64_t budget_bytes;    /* device memory pools and checkers may hold */
	uint32_t capacity[24];    /* slots per pool, by n (0: the default for n) */
	int32_t device;           /* CUDA ordinal */
	int32_t tune;             /* 1: autotune each pool shape's plan (cached per shape) */
	int32_t keep_digits;      /* 1: keep canonical residues for gfc_server_digits */
	double idle_close_s;      /* a pool with no test and nothing waiting closes after this */
} gfc_server_config;

typedef struct gfc_completion
{
	uint64_t id, nbits;
	uint32_t b, n;
	double arrival, admitted, residue_at, validated_at;  /* seconds on gfc_server_clock; validated_at < 0: unchecked */
	uint64_t res64, old64;    /* gint::isOne (src/gint.h:169-202) of the residue */
	int32_t is_prp, gl_ok;    /* gl_ok: 1 passed, 0 failed, -1 not checked */
	int32_t pool, slot, plan; /* the pool, its slot and the pool's kernel plan (gfc_batch_set_plan) */
} gfc_completion;

typedef struct gfc_server_stats
{
	uint64_t submitted, completed, pools_created, pools_open, blocks_run;
	uint64_t used_bytes, peak_bytes, budget_bytes, gl_failures;
	double open_s_sum, open_s_max;   /* seconds spent opening pools and checkers (helper threads) */
	double step_s_max;               /* longest pass of the dispatcher over its pools */
	double phase_s_max[9];           /* longest part of a pass: continuations, pools, placing, checks, closing;
	                                    of servicing a pool: event query, read-back, admission, block launch */
} gfc_server_stats;

/* block 1000, validate_group 4, budget 80 GB, default capacities, device 0,
 * tuning on, digits not kept, idle_close_s 10 (a pool also closes at once
 * when a waiting request of another size needs its memory). */
void gfc_server_default_config(gfc_server_config *cfg);

/* Starts the loop's threads; the server clock starts now. */
int gfc_server_create(const gfc_server_config *cfg, gfc_server **out);

/* Tunes the plan of the pools of size n (bases like rep_b) before requests
 * arrive, so that opening a pool later does not measure plans. */
int gfc_server_pretune(gfc_server *s, uint32_t n, uint32_t rep_b);

/* Queues a request: base b, size n (8 <= n <= 23), the exponent's nbits bits
 * (a whole test, b^(2^n), or its top bits: the state after that many
 * squarings of genefer's prp loop).  Its arrival time is now. */
int gfc_server_submit(gfc_server *s, uint64_t id, uint32_t b, uint32_t n, const uint32_t *words, uint64_t nbits);

/* Completed requests (checked, when checking is on), up to cap; waits up to
 * wait_ms for the first.  A failure of the loop is returned here. */
int gfc_server_poll(gfc_server *s, gfc_completion *out, size_t cap, size_t *got, int32_t wait_ms);

/* Canonical residue digits of a completed request (keep_digits), once. */
int gfc_server_digits(gfc_server *s, uint64_t id, int32_t *out, size_t size);

int gfc_server_get_stats(gfc_server *s, gfc_server_stats *out);
double gfc_server_clock(const gfc_server *s);

/* Stops the loop after the device work in flight; releases everything. */
void gfc_server_destroy(gfc_server *s);

/* Device bytes the server's budget counts: one pool slot of size n holding an
 * exponent of up to max_bits bits, and the root tables of size n (counted
 * once per size while a pool or checker of that size is open); the default
 * slots per pool. */
uint64_t gfc_server_slot_bytes(uint32_t n, uint64_t max_bits);
uint64_t gfc_server_table_bytes(uint32_t n);
uint32_t gfc_server_default_capacity(uint32_t n);

/* Range checks on the host: the RNS width (2 or 3) the engine picks for
 * (b, n) with one digit per coefficient, or GFC_ERR_ARG / GFC_ERR_RANGE;
 * whether b is in the packed-digit range at n (1 or 0). */
int gfc_width_for(uint32_t b, uint32_t n);
int gfc_packed_range(uint32_t b, uint32_t n);

/* ------------------------------------------------------------------ residues (host)
 * genefer's gint utilities on N host digits (src/gint.h:40-225). */

/* gint::unbalance: canonical digits in [0, b) (src/gint.h:40-102). */
void gfc_gint_unbalance(int32_t *d, size_t size, uint32_t b);

/* gint::balance: digits in (-b/2, b/2] (src/gint.h:104-149). */
void gfc_gint_balance(int32_t *d, size_t size, uint32_t b);

/* gint::isOne on canonical digits; writes res64 and old64 (src/gint.h:169-202). */
int gfc_gint_is_one(const int32_t *d, size_t size, uint32_t b, uint64_t *res64, uint64_t *old64);

/* gint::gethash64 on canonical digits (src/gint.h:204-219). */
uint64_t gfc_gint_hash64(const int32_t *d, size_t size);

#ifdef __cplusplus
}
#endif

#endif /* GFCUDA_H */
