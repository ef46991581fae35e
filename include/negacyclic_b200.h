/*
 * C ABI of the B200 negacyclic product library: c = a * b mod (X^N + 1, q).
 *
 * Every operand is N coefficients of L little-endian u32 limbs, coefficient-major
 * (coefficient i at limbs [i*L, i*L + L)), values in [0, q). q is an odd L-limb modulus
 * whose top limb is nonzero; N is a power of two from 2 to 65536.
 *
 * Each entry point returns NC_OK (0) or a negative status; nc_last_error() then returns a
 * message for the calling thread. The C++ entry points of the reference's contract
 * (fherma_init / fherma_run / fherma_free, declared in fherma.h) are exported by the same
 * library and throw std::runtime_error instead.
 */
#ifndef NEGACYCLIC_B200_H
#define NEGACYCLIC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    NC_OK = 0,
    NC_EINVAL = -1,   /* bad argument: size, alignment, modulus, null pointer */
    NC_ECUDA = -2,    /* a CUDA call failed */
    NC_ENOMEM = -3,   /* device or pinned allocation failed, or an HBM budget is exceeded */
    NC_ETIMEOUT = -4, /* a persistent-kernel dependency wait gave up (bounded spin) */
    NC_EBUSY = -5,    /* the object is in use (server full, request not finished) */
    NC_ESELFCHECK = -6 /* an init-time self-check failed (host arithmetic, tables, plan constants,
                          or the device's known-answer product) */
};

typedef struct nc_plan nc_plan;

/* Message of the last failed call on this thread ("" if none). */
const char* nc_last_error(void);

/* Library version, major * 10000 + minor * 100 + patch. */
int nc_version(void);

/* ------------------------------------------------------------------ one product per call */

/* Plan for one (N, q): tables, constants and scratch on the current device.
   Replaces fherma_init (reference fherma.h:45, solve.cu:1150-1487). W is q's bit width as
   the platform states it (L = (W + 31) / 32), or 0 to take it from q. Not reentrant: one
   product at a time per plan. */
int nc_plan_create(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, nc_plan** out);

/* The init-time checks of nc_plan_create that need no device, for one (N, q): known answers of
   the host arithmetic, the prime set and a sample of every prime's tables (once per process), then
   the plan's CRT constants: y_i (M/p_i) N = 1 mod p_i from an independent product of the other
   primes, (M/p_i mod q) p_i + ((-M) mod q) = 0 mod q for every i, the Barrett constant's defining
   inequality, and the Shoup companions; the same for the 30-bit word engine's constants where its
   primes cover the bound (y_i (M/p_i) N = 2^32 mod p_i). They hold for every valid q. Returns NC_OK, NC_EINVAL for
   an invalid point, or NC_ESELFCHECK. nc_plan_create runs the same checks and, once per device,
   an N = 8 known-answer product on the device. Mirrors the self-checks of the reference's
   fherma_init (solve.cu:1151-1165, 1285-1314, 1370-1415), without its L = 28 Barrett check,
   which rejects nearly every 868-bit q. */
int nc_self_check(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q);

/* Releases the plan (null is a no-op). Replaces fherma_free (fherma.h:47, solve.cu:1530-1567). */
int nc_plan_destroy(nc_plan* plan);

/* Host buffers in and out, synchronous. Replaces fherma_run (fherma.h:46, solve.cu:1489-1528). */
int nc_multiply(nc_plan* plan, const uint32_t* a, const uint32_t* b, uint32_t* c);

/* Device-resident operands (16-byte aligned), enqueued on `stream` exactly as given (a
   cudaStream_t; 0 is the CUDA default stream). Returns once enqueued. Uses the plan's scratch
   residues, so calls on one plan must not overlap on the device. */
int nc_multiply_device(nc_plan* plan, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, void* stream);

/* Same product as nc_multiply_device, for callers that must not allocate device memory when
   they call it (device memory owned by another framework's pool, latency-critical loops where
   cudaMalloc's implicit synchronisation is unacceptable, services that allocate only at
   start-up). It allocates nothing: the residue scratch is a fixed 8 MiB array inside the library
   (held on every GPU that loads it until exit) instead of the plan's own scratch. Limit:
   k * N <= 2^19 (N <= 16384 at an 868-bit q); larger products return NC_EINVAL. All calls share
   that array, so calls that overlap on the GPU race; nothing in it needs to start at zero. The
   array's device address is looked up (and the array loaded onto the device) when the first plan
   on that device is created, so no call of this entry point allocates, its first included. This
   entry point has no counterpart in the reference. */
int nc_multiply_device_noalloc(const nc_plan* plan, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c,
                               void* stream);

/* Chained product c = x_0 * x_1 * ... * x_{m-1} mod (X^N + 1, q) of m = 2..4 operands in one
   pass: one residue stage per operand, every forward transform and pointwise product in the row
   stage, then a single inverse transform and a single CRT. The plan's primes cover the bound of
   m canonical operands, (m - 1) log2 N + m bits(q) + 4 bits, within the same 48 primes: at
   N = 65536, m = 3 takes an 868-bit q (43 primes) and m = 4 a q of up to 731 bits; a larger q
   returns NC_EINVAL. The output
   equals the reference's pairwise products chained on the host (fherma_run twice or three times,
   solve.cu:1489-1528), with one CRT and one copy-out instead of m - 1. Such a plan also runs
   ordinary two-operand products (nc_multiply, batches, servers) with its larger prime set.
   nc_plan_factors returns m (2 for nc_plan_create). x points to m operand pointers. */
int nc_plan_create_chain(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int factors, nc_plan** out);
int nc_plan_factors(const nc_plan* plan);
/* Host operands, synchronous (the nc_multiply contract). */
int nc_multiply_chain(nc_plan* plan, const uint32_t* const* x, uint32_t* c);
/* Device operands (16-byte aligned), enqueued on `stream` (the nc_multiply_device contract). */
int nc_multiply_chain_device(nc_plan* plan, const uint32_t* const* d_x, uint32_t* d_c, void* stream);

/* Engine of the CRT accumulation sum_i v_i (M/p_i mod q) on the plan's plain path (the counterpart
   of fast_crt_kernel's 34-limb multiply-adds, solve.cu:752-836):
     NC_CRT_TC_I8  the default when the plan has at most 32 primes (q up to about 960 bits): an exact
                   u8 x u8 contraction of the bytes of v_i with a per-plan table of the bytes of
                   M/p_i mod q on the tensor cores (tcgen05.mma kind::i8, s32 accumulators in tensor
                   memory), folded back into limbs with one carry pass;
     NC_CRT_IMAD   the same sum as 32-bit carry chains on the integer pipes (always available).
   Batches and servers follow the plan's engine (tensor cores for plans of at most 30 limbs).
   Both give the same integer and so the same product. Set it only while no product of the plan
   is in flight. nc_plan_get_crt_engine returns the engine in use. */
enum { NC_CRT_IMAD = 0, NC_CRT_TC_I8 = 1 };
int nc_plan_set_crt_engine(nc_plan* plan, int engine);
int nc_plan_get_crt_engine(const nc_plan* plan);

/* Waits for the plan's own stream (the one nc_multiply uses). */
int nc_plan_synchronize(nc_plan* plan);

/* N, L, number of residue primes k of the 62-bit engine (nc_plan_word_bits gives the engine in
   use and its count), and bit length of q. Any pointer may be NULL. */
int nc_plan_query(const nc_plan* plan, uint32_t* N, uint32_t* L, uint32_t* k, uint32_t* qbits);

/* Device milliseconds from the first kernel of the last nc_multiply to its last (CUDA events).
   Operand b uploads while operand a's residue stage runs, so any part of that upload not hidden
   behind it is included. */
float nc_plan_last_kernel_ms(const nc_plan* plan);

/* Per-stage device timing of the plan's products: when enabled, each product records CUDA
   events around its three kernels (residues + forward column stages; row NTTs + pointwise;
   inverse column stages + CRT). nc_plan_stage_ms returns the three durations of the last
   product once it has completed. */
int nc_plan_set_timing(nc_plan* plan, int enable);
int nc_plan_stage_ms(const nc_plan* plan, float* ms3);

/* Measured 32-bit integer multiply-add throughput of the current device in ops/s (a chain of
   mad.lo.u32 over every SM): the denominator of the IMAD roofline. Takes a few milliseconds. */
int nc_imad_peak(double* ops_per_second);

/* Residue primes of the fixed set (p = 2^62 - m, p = 1 mod 2^17), first `count` of 48. */
int nc_primes(uint64_t* out, int count);
/* The 30-bit word engine's primes (p < 2^30, p = 1 mod 2^17, descending), first `count` of 64. */
int nc_primes32(uint32_t* out, int count);

/* ------------------------------------------------------------------ residue-stage ablation
 *
 * The residue stage alone, r[i * N + n] = x_n mod p_i (canonical, natural coefficient order,
 * prime-major: k * N u64 in d_r), for the plan's k primes, by one of two engines:
 *   NC_RESIDUES_IMAD   the product path's own arithmetic: each 32-bit limb times 2^(32 l) mod p_i,
 *                      accumulated exactly in 32-bit carry chains on the integer pipes;
 *   NC_RESIDUES_TC_I8  an exact INT8 tensor-core contraction: the bytes of x_n times the bytes of
 *                      2^(8 j) mod p_i (tcgen05.mma kind::i8, s32 accumulators in tensor memory),
 *                      recombined and reduced mod p_i; at most 32 primes (q up to about 960 bits).
 * The counterpart of both in the reference is to_residues_tiled_kernel (solve.cu:533-570), which
 * also multiplies by R^2 and psi^n. This entry point runs the stage alone (no column stages), to
 * time the two engines on the same input and check that they agree; the plan's own products pick
 * theirs with nc_plan_set_residue_engine. d_x is 16-byte aligned; enqueued on `stream`. */
enum { NC_RESIDUES_IMAD = 0, NC_RESIDUES_TC_I8 = 1 };
int nc_residues(const nc_plan* plan, const uint32_t* d_x, uint64_t* d_r, int engine, void* stream);
/* After the work has finished: 1 in *gave_up if a tensor-core launch on the current device gave up
   its bounded wait for the MMA (its residues are then not written); the flag is cleared. */
int nc_residues_status(int* gave_up);

/* Engine of the residue stage of the plan's products (nc_multiply, nc_multiply_device, the chained
   products, and the plan's products in batches and servers):
     NC_RESIDUES_TC_I8  the default: the contraction above on 128-coefficient tiles, in passes of
                        16 primes (any prime count), fused with the forward column stages (k_dec_tc);
     NC_RESIDUES_IMAD   the integer-pipe residue stage (k_dec; always available).
   Both give the same residues mod p_i and so the same product. Set it only while no product of
   the plan is in flight; nc_plan_get_residue_engine returns the engine in use. */
int nc_plan_set_residue_engine(nc_plan* plan, int engine);
int nc_plan_get_residue_engine(const nc_plan* plan);

/* ------------------------------------------------------------------ tuning */

/* Row-stage tiling of the plan's plain path: row blocks of 2^log_block residues, 2^log_radix
   residues per thread per register pass, CTAs of `threads` threads. nc_row_variants lists the
   compiled configurations valid for ring degree 2^log_n as triples (log_block, log_radix,
   threads); it returns how many it wrote, or a negative status. */
int nc_row_variants(uint32_t log_n, int* triples, int max_variants);
int nc_plan_set_row_config(nc_plan* plan, int log_block, int log_radix, int threads);
int nc_plan_get_row_config(const nc_plan* plan, int* log_block, int* log_radix, int* threads);

/* Word size of the plain path's residues. 64: the 62-bit engine (primes 2^62 - m; every plan).
   32: the 30-bit engine, primes p < 2^30 with p = 1 (mod 2^17), one u32 residue each, about twice
   as many primes at a third of the instructions per butterfly; it needs a compute capability 10.0
   device (its residue and CRT stages run on the tensor cores), a product of two operands, and a
   coefficient bound within 64 such primes (q up to 948 bits at N = 65536). It is the default
   where it can run (NC_WORD_BITS=64 in the environment keeps the 62-bit engine), the autotuner
   keeps the faster of the two, and it is in use only while both tensor-core stages are selected
   (nc_plan_set_residue_engine / nc_plan_set_crt_engine to the integer pipes select the 62-bit
   engine). Row configurations (nc_plan_set_row_config / get) apply to the engine in use;
   nc_row_variants32 lists the 30-bit engine's as nc_row_variants lists the 62-bit one's. Batches,
   servers, chained products and nc_multiply_device_noalloc run the 62-bit engine.
   nc_plan_word_bits returns 32 or 64 (the engine in use) and writes its prime count to k (may be
   NULL); nc_plan_set_word_bits fails with NC_EINVAL where the 30-bit engine cannot run. Both
   engines give the same product. Set it only while no product of the plan is in flight. */
int nc_row_variants32(uint32_t log_n, int* triples, int max_variants);
int nc_plan_set_word_bits(nc_plan* plan, int bits);
int nc_plan_word_bits(const nc_plan* plan, uint32_t* k);

/* Autotuner: times every compiled row configuration for the plan's N on the device (`reps`
   products each), keeps the fastest for this plan and for later plans of the same (N, L) in
   this process, and writes its milliseconds per product to best_ms (may be NULL). */
int nc_plan_autotune(nc_plan* plan, int reps, float* best_ms);

/* ------------------------------------------------------------------ batches
 *
 * A batch runs many products, of any mix of N and q (one plan each). Products below N = 2^15:
 * the tensor-core residue items in one launch per column length, then one persistent kernel
 * launch for the row stage (per-(prime, row block) work items in a global queue, with the residue
 * items of products on the integer residue engine and dependency counters per product, bounded
 * waits), then one CRT launch per CRT engine in use (one CTA per product tile). Products of
 * N >= 2^15 run the plain path's launches with their plan's row configuration, alternating
 * between two streams so that consecutive products overlap. The counter reset and the launches
 * are captured into a CUDA graph and replayed while the batch keeps its shape. Device buffers are
 * 16-byte aligned and must stay valid until the batch has run. */

typedef struct nc_batch nc_batch;

int nc_batch_create(nc_batch** out);
int nc_batch_destroy(nc_batch* batch);
/* c = a * b (device buffers, plan's N x L limbs). */
int nc_batch_add(nc_batch* batch, nc_plan* plan, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c);
/* c = a * b with a given in the NTT domain (nc_plan_hat_words u64 words, from nc_batch_add_forward). */
int nc_batch_add_cached(nc_batch* batch, nc_plan* plan, const uint64_t* d_a_hat, const uint32_t* d_b, uint32_t* d_c);
/* a_hat = the NTT-domain form of a, for reuse as a cached operand. */
int nc_batch_add_forward(nc_batch* batch, nc_plan* plan, const uint32_t* d_a, uint64_t* d_a_hat);
int nc_batch_clear(nc_batch* batch);
/* Enqueue every product on `stream` (0: default stream); use_graph replays a captured graph. */
int nc_batch_run(nc_batch* batch, void* stream, int use_graph);
/* Waits for the last run; NC_ETIMEOUT if a dependency wait gave up. */
int nc_batch_synchronize(nc_batch* batch);
/* Products, persistent CTAs of the last run, bytes of residue scratch held. Pointers may be NULL. */
int nc_batch_query(const nc_batch* batch, uint32_t* products, uint32_t* ctas, uint64_t* scratch_bytes);
/* u64 words that hold the NTT-domain form of one operand of this plan on either engine: k * N u64
   on the 62-bit engine, k32 * N u32 on the 30-bit one (the plan's engine decides which a batch's
   forward and cached-a products use). */
uint64_t nc_plan_hat_words(const nc_plan* plan);

/* ------------------------------------------------------------------ serving
 *
 * Continuous batching. nc_server_submit copies host operands into pinned staging and returns a
 * request id (it blocks while staging is full). A scheduler thread admits queued requests in
 * arrival order while the HBM budget holds them (operands, product and residue scratch), runs
 * everything admitted as one persistent batch on the next free stream, and keeps admitting new
 * requests into further batches while earlier ones run, so their work overlaps on the device.
 * Operands registered with nc_server_register_operand stay resident in their NTT-domain form;
 * requests that name one (a = NULL, operand_id >= 0) skip its transform. nc_server_wait returns
 * the product and the request's latency from submit to result in pinned host memory. A request
 * holds its staging (3 N L u32) from submit until nc_server_wait collects it, so callers that
 * submit many requests before collecting any must size staging for all of them, or submit blocks
 * for good. */

typedef struct nc_server nc_server;

int nc_server_create(uint64_t hbm_budget_bytes, uint64_t staging_bytes, int max_batch, int streams, nc_server** out);
int nc_server_destroy(nc_server* server);
int nc_server_register_operand(nc_server* server, nc_plan* plan, const uint32_t* a, int* operand_id);
int nc_server_release_operand(nc_server* server, int operand_id);
int nc_server_submit(nc_server* server, nc_plan* plan, const uint32_t* a, int operand_id, const uint32_t* b,
                     uint64_t* request_id);
/* 1 when the request is finished (nc_server_wait returns at once), 0 while pending. */
int nc_server_poll(nc_server* server, uint64_t request_id);
int nc_server_wait(nc_server* server, uint64_t request_id, uint32_t* c, double* latency_ms);
/* Latency percentiles over completed requests, their count, completed products per second
   since the first submit, device bytes in use, batches launched, batches whose bounded
   dependency wait gave up (their requests fail with NC_ETIMEOUT). Pointers may be NULL. */
int nc_server_stats(nc_server* server, double* p50_ms, double* p99_ms, uint64_t* completed, double* products_per_s,
                    uint64_t* hbm_in_use, uint64_t* batches, uint64_t* timeouts);
/* Where the served time goes: bytes copied host -> device and device -> host by finished batches;
   on the device's clock, the time during which at least one batch had copies or kernels in flight
   (the union of the batches' intervals from first copy to last copy) within the window from the
   first batch's start to the last batch's end; and the host time the scheduler thread spent
   enqueueing batches. Pointers may be NULL. No counterpart in the reference, which serves
   nothing. */
int nc_server_io_stats(nc_server* server, uint64_t* h2d_bytes, uint64_t* d2h_bytes, double* device_busy_ms,
                       double* device_window_ms, double* scheduler_ms);

#ifdef __cplusplus
}
#endif

#endif /* NEGACYCLIC_B200_H */
