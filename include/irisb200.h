/*
 * irisb200 -- C ABI of the B200 iris uniqueness hot path.
 *
 * The three MPC parties of worldcoin/iris-mpc run co-resident on one GPU.
 * Each party has its own CUDA stream and memory pool; a message from one
 * party to the next is a device-buffer handoff on that GPU instead of an NCCL
 * send/recv.  Every entry point returns 0 on success or a negative irs_status
 * (it never aborts); irs_last_error() describes the last failure of the
 * calling thread.  Handles are opaque; host buffers are caller-owned; device
 * buffers are library-owned unless a function says otherwise.  Streams are
 * passed as void* (cudaStream_t); NULL means the party's own stream.
 *
 * Each declaration names the reference interface it replaces (file:line in
 * worldcoin/iris-mpc).
 */
#ifndef IRISB200_H
#define IRISB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum irs_status {
  IRS_OK = 0,
  IRS_ERR_INVALID = -1,    /* bad argument or shape */
  IRS_ERR_CUDA = -2,       /* CUDA runtime error */
  IRS_ERR_NOMEM = -3,      /* device allocation failed */
  IRS_ERR_STATE = -4,      /* call out of order (e.g. dot before query upload) */
  IRS_ERR_DEVICE = -5,     /* a kernel reported an error (bounded wait expired) */
  IRS_ERR_OVERFLOW = -6,   /* a result list exceeded its capacity */
};

#define IRS_IRIS_CODE_LENGTH 12800 /* iris-mpc-common/src/lib.rs:15 */
#define IRS_MASK_CODE_LENGTH 6400  /* iris-mpc-common/src/lib.rs:16 */
#define IRS_ROTATIONS 31           /* iris-mpc-common/src/lib.rs:17 */
#define IRS_SLOT_ROWS 32           /* query rows per query iris: 31 rotations + 1 pad row */
#define IRS_MAX_MATCHES_LEN 256    /* iris-mpc-gpu/src/dot/distance_comparator.rs:26 */
#define IRS_THRESHOLD_A 20316u     /* iris-mpc-gpu/src/dot/mod.rs:12 (ratio 0.345) */
#define IRS_THRESHOLD_ANON_STATS_A 16384u /* iris-mpc-gpu/src/dot/mod.rs:14 (ratio 0.375) */

/* Last error message of the calling thread ("" if none). */
const char* irs_last_error(void);
/* Library build string (architecture, version). */
const char* irs_version(void);

/* ------------------------------------------------------------------------ */
/* Device manager: one GPU hosting the three parties.                        */
/* Replaces DeviceManager::init / fork_streams / split_into_n_chunks          */
/* (iris-mpc-gpu/src/helpers/device_manager.rs:28-157) and the NCCL ring of   */
/* NcclComm (iris-mpc-gpu/src/helpers/comm.rs:8-270,                          */
/* device_manager.rs:289-344): party p sends to (p+1)%3 and receives from     */
/* (p+2)%3 through device buffers.                                            */
/* ------------------------------------------------------------------------ */
typedef struct irs_device_manager irs_device_manager;

int irs_device_manager_init(int device, irs_device_manager** out);
int irs_device_manager_destroy(irs_device_manager* dm);
/* The CUDA stream of party `party` (0..2). */
int irs_device_manager_stream(irs_device_manager* dm, int party, void** stream);
/* Synchronise all party streams (DeviceManager::await_streams). */
int irs_device_manager_synchronize(irs_device_manager* dm);
/* Device error word: 0, or the code of the first bounded wait that expired. */
int irs_device_manager_error(irs_device_manager* dm, int* code);
int irs_device_manager_clear_error(irs_device_manager* dm);
/* Error codes of the device error word. */
#define IRS_DEV_ERR_TIMEOUT_FULL 1      /* the GEMM's MMA waited too long for a TMA stage */
#define IRS_DEV_ERR_TIMEOUT_EMPTY 2     /* the GEMM's loader waited too long for a free stage */
#define IRS_DEV_ERR_TIMEOUT_ACC_FULL 3  /* the GEMM's epilogue waited too long for its accumulator */
#define IRS_DEV_ERR_TIMEOUT_ACC_EMPTY 4 /* the GEMM's MMA waited too long for the epilogue */
#define IRS_DEV_ERR_TIMEOUT_DRAIN 5     /* an exit-time wait for in-flight copies gave up */
/* Test hook of the failure path (the reference panics on a stuck NCCL or
 * kernel wait, helpers/device_manager.rs:25-26,330-343, under panic = abort):
 * the next dot launch of this device manager runs with `wait_limit_ns` as its
 * bounded-wait limit (1 us .. 10 s; the default is 2 s) and its first CTA
 * issues no loads, so that CTA's MMA stage wait runs out.  The kernel records
 * IRS_DEV_ERR_TIMEOUT_FULL in the device error word and returns (no memory
 * access is skipped or added elsewhere; the other CTAs finish their tiles);
 * the next synchronising call returns IRS_ERR_DEVICE, the device stays usable,
 * and irs_device_manager_clear_error resets the word.  One shot; refused
 * during a graph capture. */
int irs_device_manager_test_stall_next_dot(irs_device_manager* dm, uint64_t wait_limit_ns);
/* Device-resident batch counter (the reference advances host-side ChaCha
 * counters instead, ChachaCommon::advance_counter, rng/chacha.rs:32-36):
 * engines and circuits switched to it with
 * irs_sharedb_use_batch_counter / irs_circuits_use_batch_counter read their
 * ChaCha batch id from device memory at run time, so a captured graph can be
 * replayed for every batch with a fresh counter (set here, outside capture). */
int irs_device_manager_set_batch_counter(irs_device_manager* dm, uint64_t batch_id, void* stream);
/* Advances the device batch counter on the stream (b -> b mod (2^24 - 1) + 1)
 * without a host round trip: a serving loop that launches one DB chunk per
 * step draws fresh randomness for every step while the host runs ahead. */
int irs_device_manager_advance_batch_counter(irs_device_manager* dm, void* stream);
/* Stage timers (the reference's record_stream_time! / log_timers behind
 * enable_debug_timing, server/actor.rs:71-85,2887-2911): while on, every dot
 * launch ("dot") and threshold/open launch ("threshold_open") outside a graph
 * capture is bracketed by CUDA events on its stream.  irs_device_manager_timings
 * waits for them and writes "label=ms/launches;..." (summed since the last
 * reset) into buf; reset != 0 clears the sums. */
int irs_device_manager_set_timing(irs_device_manager* dm, int on);
int irs_device_manager_timings(irs_device_manager* dm, char* buf, size_t cap, int reset);
/* Reads the device batch counter (after the work queued on party 0's stream):
 * with the parties' seeds and the DB length it is the whole randomness state
 * to checkpoint (ChaChaCtx is (seed, counter), rng/chacha.rs:205-250). */
int irs_device_manager_get_batch_counter(irs_device_manager* dm, uint64_t* batch_id);
/* Number of SMs the persistent kernels size their grids to. */
int irs_device_manager_sm_count(irs_device_manager* dm, int* n);
/* Host synchronisation of the calls that take host buffers (default on; no
 * counterpart in the reference, whose calls are stream-ordered cudarc copies).
 * With it off, irs_sharedb_query_put_base, irs_sharedb_query_expand_rows,
 * irs_sharedb_query_upload_rows, irs_sharedb_gather_records,
 * irs_dc_set_segments, irs_dc_take_rows, irs_dc_fetch_rows and
 * irs_dc_fetch_final_results return as soon as their copies and kernels are
 * enqueued: their host buffers must then be page-locked
 * (irs_host_alloc_pinned) and stay unchanged until the work has run, and the
 * outputs of the last three are valid after an event recorded behind them on
 * the party-0 stream has completed (device
 * errors: irs_device_manager_error).  A serving loop or a batched caller uses
 * this to prepare and launch batch k+1 while batch k runs. */
int irs_device_manager_set_host_sync(irs_device_manager* dm, int on);
/* CUDA events for the asynchronous mode (cudaEventDisableTiming); the
 * reference uses raw CUevents through cudarc (device_manager.rs). */
int irs_event_create(void** ev);
int irs_event_record(void* ev, void* stream);
int irs_event_synchronize(void* ev);
/* *done = 1 when the work before the event has completed, else 0. */
int irs_event_query(void* ev, int* done);
int irs_event_destroy(void* ev);
/* Free and total device memory (cudaMemGetInfo), for admission by free HBM
 * (no counterpart: the reference sizes its batches statically). */
int irs_device_manager_mem_info(irs_device_manager* dm, size_t* free_bytes, size_t* total_bytes);

/* Plain device memory helpers for callers that stage their own buffers. */
int irs_device_alloc(irs_device_manager* dm, size_t bytes, void** ptr);
/* Page-locked host memory (register_host_memory, device_manager.rs:214-238). */
int irs_host_alloc_pinned(size_t bytes, void** ptr);
int irs_host_free_pinned(void* ptr);
int irs_device_free(irs_device_manager* dm, void* ptr);
int irs_copy_h2d(void* dst, const void* src, size_t bytes, void* stream);
int irs_copy_d2h(void* dst, const void* src, size_t bytes, void* stream);
int irs_stream_synchronize(void* stream);

/* ------------------------------------------------------------------------ */
/* ShareDB: one party's dot-product engine over a device-resident share DB.   */
/* (iris-mpc-gpu/src/dot/share_db.rs:448-1070)                               */
/* ------------------------------------------------------------------------ */
typedef struct irs_sharedb irs_sharedb;

/* ShareDB::init (share_db.rs:467-573).  code_length: 12800 (codes) or 6400
 * (trimmed masks).  query_length: query rows per batch (padded internally to
 * a multiple of 64).  seed0 = this party's own ChaCha seed, seed1 = the
 * previous party's seed; is_remote = 0 disables the zero-share mask (the
 * reference's empty `comms`). */
int irs_sharedb_init(irs_device_manager* dm, int peer_id, size_t max_db_length, size_t query_length,
                     size_t code_length, const uint32_t seed0[8], const uint32_t seed1[8], int is_remote,
                     irs_sharedb** out);
int irs_sharedb_destroy(irs_sharedb* db);
/* ShareDB::alloc_db (share_db.rs:575-618); the DB lives in HBM. */
int irs_sharedb_alloc_db(irs_sharedb* db, size_t max_db_length);
/* ShareDB::load_single_record_from_db for records first..first+n-1
 * (share_db.rs:620-655): u16 share coefficients [n][code_length]. */
int irs_sharedb_load_records(irs_sharedb* db, size_t first, size_t n, const uint16_t* records);
/* ShareDB::load_single_record_from_s3 (share_db.rs:657-684): the stored i8
 * limbs (byte - 128), [n][code_length] each. */
int irs_sharedb_load_records_i8(irs_sharedb* db, size_t first, size_t n, const uint8_t* limb0,
                                const uint8_t* limb1);
/* Reads records first..first+n-1 back as u16 coefficients [n][code_length]
 * (the inverse of load_records; CudaVec2DSlicer limb planes,
 * iris-mpc-gpu/src/helpers/query_processor.rs:20-60). */
int irs_sharedb_fetch_records(irs_sharedb* db, size_t first, size_t n, uint16_t* records);
/* Number of valid records (SlicedProcessedDatabase db_lens). */
int irs_sharedb_set_db_len(irs_sharedb* db, size_t len);
int irs_sharedb_db_len(irs_sharedb* db, size_t* len);
/* Fills records first..first+n-1 of the six engines (party p code/mask) with
 * the seeded synthetic irises of the benchmark workload (device-side). */
int irs_sharedb_synth_db(irs_sharedb* const code_engines[3], irs_sharedb* const mask_engines[3], uint64_t seed,
                         size_t first, size_t n);

/* Records 0..n-1 of one engine filled with seeded uniform limb bytes (a
 * single-engine benchmark DB: the GEMM sweep of matmul.rs has no encoding). */
int irs_sharedb_fill_random(irs_sharedb* db, uint64_t seed, size_t n);
/* Seeded uniform bytes in a device buffer (8-byte aligned, bytes % 8 == 0);
 * benchmark inputs, no counterpart in the reference. */
int irs_device_fill_random(void* ptr, size_t bytes, uint64_t seed, void* stream);

/* preprocess_iris_code_query_share / preprocess_mask_code_query_share
 * (galois_engine.rs:23-40,193-195,438-440) on the host, in place: each GR4
 * block times the party's Lagrange coefficient at 0, converted to basis B. */
int irs_preprocess_query_share(int party, uint16_t* coefs, size_t n);

/* encode_iris_code / encode_mask_code (galois_engine.rs:319-397) of one iris
 * (host): code_bits / mask_bits are the 12800 plaintext bits as u64 words
 * [200] (bit i of the iris = bit i % 64 of word i / 64), seed drives the
 * sharing randomness.  Writes the three parties' shares, code_out [3][12800]
 * and the trimmed mask_out [3][6400]: DB records when preprocess = 0, query
 * shares (irs_preprocess_query_share applied) otherwise.  A deletion writes
 * the encoding of the default iris (all-zero code, full mask; the reference's
 * get_dummy_shares_for_deletion, iris_db/mod.rs:10-23) over the record. */
int irs_encode_iris(const uint64_t* code_bits, const uint64_t* mask_bits, uint64_t seed, int preprocess,
                    uint16_t* code_out, uint16_t* mask_out);
/* Seeded synthetic queries of the benchmark workload (host): query j is a
 * near-duplicate of DB entry planted_entry[j] (code bits flipped with p = 0.2,
 * rotated by planted_rot[j] columns) or, for planted_entry[j] < 0, a fresh
 * iris.  Writes the three parties' shares, code_out [3][n_queries][12800] and
 * mask_out [3][n_queries][6400] (trimmed), preprocessed when `preprocess`.
 * The DB entries are those irs_sharedb_synth_db generates for db_seed. */
int irs_synth_queries(uint64_t db_seed, uint64_t q_seed, size_t n_queries, const int64_t* planted_entry,
                      const int32_t* planted_rot, int preprocess, uint16_t* code_out, uint16_t* mask_out);

/* Query upload: preprocess_query + htod_transfer_query
 * (share_db.rs:45-59; device_manager.rs:159-212), rows given as-is
 * [n_rows][code_length] (already Lagrange-preprocessed and rotated). */
int irs_sharedb_query_upload(irs_sharedb* db, const uint16_t* rows, size_t n_rows);

/* Query slot: 32 query rows holding rotations rot_lo..rot_lo+n_rot-1 of base
 * query `src` (rotation index 15 = centre, all_rotations(),
 * galois_engine.rs:197-206), reported as bitmap row `query`. */
typedef struct irs_query_slot {
  uint32_t src;
  uint32_t rot_lo;
  uint32_t n_rot;
  uint32_t query;
} irs_query_slot;

/* Uploads preprocessed base query shares [n_base][code_length] and expands
 * the rotations on the device into 32-row slots (row 32*s + r). */
int irs_sharedb_query_upload_slots(irs_sharedb* db, const uint16_t* base, size_t n_base,
                                   const irs_query_slot* slots, size_t n_slots);
/* Uploads preprocessed base queries [n_base][code_length] and fills query row
 * r with row_desc[r] = (src << 8) | (mirror << 7) | rotation (rotation 0..30
 * of base query src, 15 = centre; mirror = 1: of its mirrored form, the
 * reference's mirrored_code / mirrored_mask, galois_engine.rs:218-225,520-543,
 * applied on the device), 0xFFFFFFFF = zero row.  Packs queries with any
 * rotation count densely (the batched launch of uneven requests); a request
 * and its mirror share one base.  No counterpart in the reference, which
 * gives every query a block of 31 rotation rows (htod_transfer_query,
 * device_manager.rs:159-212) and mirrors on the host. */
int irs_sharedb_query_upload_rows(irs_sharedb* db, const uint16_t* base, size_t n_base, const uint32_t* row_desc,
                                  size_t n_rows);
/* Resident base-query pool for a serving loop (no counterpart in the
 * reference, whose actor uploads every batch whole): writes preprocessed base
 * queries [first, first + n) of the pool (the query staging area) without
 * touching the others, so a request admitted while others are in flight costs
 * one upload of its own shares. */
int irs_sharedb_query_put_base(irs_sharedb* db, size_t first, size_t n, const uint16_t* base);
/* irs_sharedb_query_upload_rows over the resident pool [0, n_base): rebuilds
 * the query rows from the row table alone. */
int irs_sharedb_query_expand_rows(irs_sharedb* db, size_t n_base, const uint32_t* row_desc, size_t n_rows);
/* prefetch_subset (share_db.rs:344-407), device to device: copies DB records
 * ids[k] of `src` into records k of `dst` (same party and code length) and
 * sets dst's length to n.  Used for reauth targets and subset re-checks. */
int irs_sharedb_gather_records(irs_sharedb* dst, irs_sharedb* src, const uint32_t* ids, size_t n);
/* mirrored_code / mirrored_mask (galois_engine.rs:218-225,520-543) of a
 * (preprocessed or raw) query share, in place; flip_imaginary = 1 for codes. */
int irs_mirror_query_share(uint16_t* coefs, size_t n, int flip_imaginary);
/* Tile width of the dot kernel along the query rows: 64, 128 or 256, or 0 for
 * the library's choice (the batch autotuner's knob; no counterpart in the
 * reference, where cuBLAS picks its own tiles).  The padded row count of a
 * batch is its uploaded rows rounded up to 64, and further to 128 (up to 768
 * rows) or 256 (above) when the query capacity allows; the extra rows are zero.
 * Default: the 128-row tile up to 768 padded rows, else the 256-row tile. */
int irs_sharedb_set_tile(irs_sharedb* db, int block_n);
/* on != 0: the 256-row tile runs as the two-SM GEMM (a cluster of two CTAs
 * with tcgen05.mma.cta_group::2 on a 256-entry x 256-row tile; same results).
 * Off by default: under the B200's power cap it trades clock for MAC rate, so
 * the batch autotuner decides (no counterpart in the reference). */
int irs_sharedb_set_pair(irs_sharedb* db, int on);
int irs_sharedb_use_batch_counter(irs_sharedb* db, int on);
/* Starts a new batch: the zero-share mask and circuit keystreams are drawn at
 * ChaCha counter (batch_id << 40) | position (ChaChaCtx counter,
 * iris-mpc-gpu/src/rng/chacha.rs:205-250). */
int irs_sharedb_set_batch(irs_sharedb* db, uint64_t batch_id);

/* ShareDB::dot + dot_reduce_and_multiply (share_db.rs:800-905) fused:
 * entries [offset, offset+len) against the uploaded queries; result shares
 * (multiplier * dot + ks_own - ks_prev mod 2^16) stay on the device.
 * offset must be a multiple of 32. */
int irs_sharedb_dot(irs_sharedb* db, size_t offset, size_t len, uint16_t multiplier, void* stream);
/* The same for several engines in one launch (e.g. 3 parties x code/mask);
 * multipliers[i] per engine; stream NULL = party 0's stream. */
int irs_sharedb_dot_many(irs_sharedb* const* engines, const uint16_t* multipliers, int n, size_t offset,
                         size_t len, void* stream);
/* ShareDB::fetch_results (share_db.rs:1038-1048): the party's own result
 * share in the reference layout [query_length][len]. */
int irs_sharedb_fetch_results(irs_sharedb* db, uint16_t* host, size_t len);
/* ShareDB::result_chunk_shares (share_db.rs:1050-1069): device pointer to the
 * party's own share, layout [entry][row_stride] (entry-major).  The replicated
 * `b` share of party p is party (p+2)%3's own share (reshare_results,
 * share_db.rs:1004-1036, becomes this handoff). */
int irs_sharedb_result_view(irs_sharedb* db, const uint16_t** dev, size_t* row_stride);

/* ------------------------------------------------------------------------ */
/* Circuits: the threshold protocol of the three parties.                    */
/* (iris-mpc-gpu/src/threshold_ring/protocol.rs:433-2611)                    */
/* ------------------------------------------------------------------------ */
typedef struct irs_circuits irs_circuits;

/* Circuits::new for the three parties (protocol.rs:463-514).
 * seeds[p] = party p's (seed0, seed1); seed1 of party p must equal seed0 of
 * party (p+2)%3 (the correlated-randomness ring). */
int irs_circuits_new(irs_device_manager* dm, const uint32_t seeds[3][2][8], irs_circuits** out);
int irs_circuits_destroy(irs_circuits* c);
int irs_circuits_set_batch(irs_circuits* c, uint64_t batch_id);
int irs_circuits_use_batch_counter(irs_circuits* c, int on);

/* compare_threshold_masked_many (protocol.rs:2519-2546) on n elements
 * (multiple of 64).  code_a[p]/mask_a[p]: party p's own u16 share (device);
 * party p's second share is party (p+2)%3's own.  res_a[p]/res_b[p]:
 * device u64 words (n/64) receiving party p's replicated share of the match
 * bit (bit i of word w = element 64w + i); either may be NULL.  opened:
 * optional device u64 words receiving the opened bits. */
int irs_circuits_compare_threshold_masked_many(irs_circuits* c, const uint16_t* const code_a[3],
                                               const uint16_t* const mask_a[3], size_t n, uint32_t threshold_a,
                                               uint64_t* const res_a[3], uint64_t* const res_b[3], uint64_t* opened,
                                               void* stream);
/* compare_threshold_masked_many for callers that cannot allocate device
 * memory after start-up (e.g. a server that reserved all of HBM for the share
 * database, or a host runtime whose own allocator owns the device).  No
 * counterpart in the reference.  Same arguments and results as
 * irs_circuits_compare_threshold_masked_many, but its scratch lives in a
 * static device array of IRS_NOALLOC_MAX_ELEMENTS / 32 words per party that
 * every GPU loading the library holds until exit; it calls no allocator.
 * n above IRS_NOALLOC_MAX_ELEMENTS is rejected with IRS_ERR_INVALID.  A call
 * outside stream capture looks up the array's device address
 * (cudaGetSymbolAddress, so it stays right after a cudaDeviceReset); a call
 * inside a capture reuses the address of the device's last call outside one,
 * so make the first call on each device before any stream capture
 * (IRS_ERR_STATE otherwise).  All calls share the array: calls whose work
 * overlaps on the GPU race and must be serialised by the caller. */
#define IRS_NOALLOC_MAX_ELEMENTS (1u << 22)
int irs_circuits_compare_threshold_masked_many_noalloc(irs_circuits* c, const uint16_t* const code_a[3],
                                                       const uint16_t* const mask_a[3], size_t n,
                                                       uint32_t threshold_a, uint64_t* const res_a[3],
                                                       uint64_t* const res_b[3], uint64_t* opened, void* stream);
/* lift_mul_sub + extract_msb with the lifted mask at zero
 * (tests/extract_msb_mod.rs:180-215): msb of -code*2^16 - 1. */
int irs_circuits_extract_msb_of_code(irs_circuits* c, const uint16_t* const code_a[3], size_t n,
                                     uint64_t* const res_a[3], uint64_t* const res_b[3], uint64_t* opened,
                                     void* stream);
/* or_reduce_result / or_tree_on_gpu (threshold_ring/protocol.rs:2363-2515):
 * the shared OR of all n result bits (n a multiple of 64), given every party's
 * a-share res_a[p] (u64 words, as compare_threshold_masked_many writes them;
 * party p's b-share is party p-1's a-share).  AND gates on each party's own
 * view, the reference's halving tree over words, then a collapse of the last
 * word's 32 bits.  Writes host out[0..2] = party p's a-share of the OR bit,
 * out[3] = the opened bit.  Synchronous. */
int irs_circuits_or_reduce(irs_circuits* c, const uint64_t* const res_a[3], size_t n, uint32_t out[4],
                           void* stream);
/* compare_threshold_masked_many_with_or_tree (protocol.rs:2594-2610): the
 * threshold comparison of n elements followed by the OR tree; out as above. */
int irs_circuits_compare_threshold_masked_many_with_or_tree(irs_circuits* c, const uint16_t* const code_a[3],
                                                            const uint16_t* const mask_a[3], size_t n,
                                                            uint32_t threshold_a, uint32_t out[4], void* stream);
/* lift_mpc (protocol.rs:2041-2074): per party p, corr[p] receives two u16
 * arrays of n (party p's own component of the injected carries c1, c2);
 * sum_p mask_p - (sum corr1 << 16) - (sum corr2 << 17) = mask in Z_2^32. */
int irs_circuits_lift_mpc(irs_circuits* c, const uint16_t* const mask_a[3], size_t n, uint16_t* const corr[3],
                          void* stream);

/* ------------------------------------------------------------------------ */
/* DistanceComparator: opening, rotation OR, candidate lists and merges.     */
/* (iris-mpc-gpu/src/dot/distance_comparator.rs:28-894)                      */
/* ------------------------------------------------------------------------ */
typedef struct irs_distance_comparator irs_distance_comparator;

/* DistanceComparator::init (distance_comparator.rs:58-190). */
int irs_dc_init(irs_device_manager* dm, size_t max_queries, size_t max_db_length, size_t match_list_cap,
                irs_distance_comparator** out);
int irs_dc_destroy(irs_distance_comparator* dc);
/* Clears bitmaps, counters and final results for a new batch. */
int irs_dc_reset(irs_distance_comparator* dc, void* stream);

/* The hot step of compare_query_against_db_and_self_prefiltering
 * (iris-mpc-gpu/src/server/actor.rs:2405-2519): for the six engines' current
 * results over entries [offset, offset+len), runs the threshold protocol,
 * opens the bits (open, actor.rs:2928-2997), ORs every slot's valid rotation
 * rows (openResults, dot/kernel.cu:54-116) into the match bitmap and appends
 * (query, entry) pairs to the match list.  slot_valid[s]: bit mask of valid
 * rows of slot s (NULL = rows 0..30); slot_query[s]: bitmap row of slot s
 * (NULL = s).  `self_check` != 0 writes the batch-self bitmap instead. */
int irs_dc_compare_threshold_open(irs_distance_comparator* dc, irs_circuits* c, irs_sharedb* const code_engines[3],
                                  irs_sharedb* const mask_engines[3], size_t offset, size_t len, size_t n_slots,
                                  const uint32_t* slot_valid, const uint32_t* slot_query, uint32_t threshold_a,
                                  int self_check, void* stream);
/* Segment table for packed query rows (no counterpart in the reference, one
 * query per 31 rows there): slot s (32 rows) holds segments
 * seg_start[s] .. seg_start[s+1]-1; segment k ORs the opened bits of rows
 * seg_mask[k] into bitmap row seg_query[k].  Copied to the device once, so the
 * prepared call below can run inside a captured CUDA graph. */
int irs_dc_set_segments(irs_distance_comparator* dc, size_t n_slots, const uint32_t* seg_start,
                        const uint32_t* seg_query, const uint32_t* seg_mask);
/* irs_dc_compare_threshold_open with the stored segment table; performs no
 * host synchronisation (graph-capturable). */
int irs_dc_compare_threshold_open_prepared(irs_distance_comparator* dc, irs_circuits* c,
                                           irs_sharedb* const code_engines[3], irs_sharedb* const mask_engines[3],
                                           size_t offset, size_t len, uint32_t threshold_a, int self_check,
                                           void* stream);
/* The six limb GEMMs (irs_sharedb_dot_many with multipliers {1,1,1,2,2,2})
 * and irs_dc_compare_threshold_open over entries [offset, offset+len) in ONE
 * persistent kernel: per 128-entry x 128-row tile the six engines' masked dot
 * shares go to an L2-resident ring slot of the CTA (never to the engines'
 * result buffers) and the same CTA runs the threshold, open and rotation OR
 * on them (the reference's per-chunk Phase 1 + Phase 2 + open,
 * iris-mpc-gpu/src/server/actor.rs:2376-2519).  Plain slots (use_segments = 0:
 * n_slots 32-row slots, rows 0..30 valid, slot s reported as query s) or the
 * stored segment table (use_segments = 1, n_slots ignored).  Results equal the
 * two-launch path's bit for bit.  Needs the padded query rows in multiples of
 * 128.  The first call allocates the comparator's ring (n_SMs x 196,608
 * bytes; a call with len = 0 only allocates), so make it before any graph
 * capture; later calls are graph-capturable.  The ring belongs to the
 * comparator: two scans of one comparator must not overlap on the GPU (issue
 * them on one stream, as all of a comparator's calls).  Afterwards the
 * engines hold no dot shares (irs_sharedb_fetch_results refuses). */
int irs_dc_scan_fused(irs_distance_comparator* dc, irs_circuits* c, irs_sharedb* const code_engines[3],
                      irs_sharedb* const mask_engines[3], size_t offset, size_t len, size_t n_slots,
                      uint32_t threshold_a, int use_segments, void* stream);
/* Match lists of selected bitmap rows (the per-query assembly of
 * fetch_final_results, distance_comparator.rs, for rows chosen by the caller):
 * counts[i] = set bits of row rows[i] below db_len, ids [n][IRS_MAX_MATCHES_LEN]
 * = the lowest min(counts[i], 256) of those entries in ascending order.  With
 * clear != 0 the rows are zeroed in the same pass (a serving loop reusing the
 * rows of completed requests).  Synchronous. */
int irs_dc_take_rows(irs_distance_comparator* dc, const uint32_t* rows, size_t n, size_t db_len, int clear,
                     uint32_t* counts, uint32_t* ids);
/* Anonymised-statistics distance capture (openResults' match distance
 * buffers, iris-mpc-gpu/src/dot/kernel.cu:73-106; DistanceCache,
 * server/anon_stats.rs): once enabled, every later compare_threshold_open(_prepared)
 * of this comparator appends, for each opened match of a valid query row, the
 * DB entry, the query row (32 * slot + row of the slot) and the three parties'
 * additive components of the code and (x2) mask dot shares, up to `cap`
 * records (further matches are counted, not stored).  Run it on the prefilter
 * pass (IRS_THRESHOLD_ANON_STATS_A) as the reference does. */
int irs_dc_enable_distance_capture(irs_distance_comparator* dc, size_t cap);
/* Pairs (bitmap row query[i], DB entry entry[i]) whose distances are captured
 * for every valid query row whether or not they match (openResults'
 * anon_stats_idx, kernel.cu:73-86: the reauth targets); n <= 256, replaces the
 * previous list, n = 0 clears it.  Needs the capture enabled. */
int irs_dc_set_forced_distances(irs_distance_comparator* dc, const uint32_t* query, const uint32_t* entry, size_t n);
/* Copies up to `cap` captured records: entry [cap], row [cap], code [3][cap],
 * mask [3][cap] (component p at p * cap); *n = records captured so far
 * (possibly above the capture capacity).  reset != 0 empties the capture. */
int irs_dc_fetch_distances(irs_distance_comparator* dc, size_t cap, uint32_t* entry, uint32_t* row, uint16_t* code,
                           uint16_t* mask, size_t* n, int reset);
/* Clears bitmap rows [first, first + n) (a query row reused by the serving
 * loop for a new request; no counterpart in the reference). */
int irs_dc_clear_rows(irs_distance_comparator* dc, size_t first, size_t n, void* stream);
/* Bitmap rows [first, first + n) in the internal layout: u32 words
 * [n][row_words], bit j of word w = entry 32w + j; *row_words receives the
 * words per row (the bitmap stride). */
int irs_dc_fetch_rows(irs_distance_comparator* dc, size_t first, size_t n, uint32_t* host, size_t cap_words,
                      size_t* row_words);
/* Match bitmap in the reference layout: bit (q * db_len + e) set if query q
 * matches entry e (u64 words, ceil(n_queries * db_len / 64)). */
int irs_dc_fetch_bitmap(irs_distance_comparator* dc, size_t n_queries, size_t db_len, uint64_t* host);
/* Matches (query, entry) pairs appended since the last reset. */
int irs_dc_fetch_matches(irs_distance_comparator* dc, uint32_t* pairs, size_t cap, size_t* n);
/* get_partial_results (distance_comparator.rs:545-646, partialDbResults):
 * sorted unique entry indices matched by any query; *n may exceed cap
 * (overflow is reported as IRS_ERR_OVERFLOW after filling cap ids). */
int irs_dc_get_partial_results(irs_distance_comparator* dc, size_t n_queries, size_t db_len, uint32_t* ids,
                               size_t cap, size_t* n);
/* join_db_matches(_with_bitmaps) (distance_comparator.rs:688-729): merges the
 * DB bitmap of this comparator (left eye) with `right` (NULL: single eye) and
 * an optional OR-policy bitmap (device, same layout as the internal bitmap);
 * final results per query = smallest matched entry. */
int irs_dc_join_db_matches(irs_distance_comparator* dc, irs_distance_comparator* right, const uint32_t* or_policy,
                           size_t n_queries, size_t db_len, void* stream);
/* join_batch_matches (distance_comparator.rs:731-746, mergeBatchResults). */
int irs_dc_join_batch_matches(irs_distance_comparator* dc, irs_distance_comparator* right, size_t n_queries,
                              void* stream);
/* fetch_final_results / fetch_match_counters / fetch_all_match_ids
 * (distance_comparator.rs:748-893): final[q] = smallest matched entry,
 * 0xFFFFFFFE for an in-batch duplicate, 0xFFFFFFFF for no match.  In the
 * asynchronous host mode the copies are only enqueued on party 0's stream
 * (page-locked outputs, valid once an event recorded after the call has
 * completed). */
int irs_dc_fetch_final_results(irs_distance_comparator* dc, size_t n_queries, uint32_t* final_results,
                               uint32_t* match_counters, uint32_t* all_matches);

/* ------------------------------------------------------------------------ */
/* The plain DB pass and its autotuner: the chunk loop of                    */
/* compare_query_against_db_and_self_prefiltering (actor.rs:2246-2589) over  */
/* the resident engines for one uploaded batch of n_slots 32-row query slots */
/* (rows 0..30 valid, slot s reported as query s) and entries [0, db_len).   */
/* Per chunk one of three paths: the limb GEMM launch then the threshold     */
/* launch (IRS_SCAN_SPLIT, at a tile width), the same with the two-SM GEMM   */
/* (IRS_SCAN_PAIR, 256-row tile), or irs_dc_scan_fused (IRS_SCAN_FUSED).     */
/* Results are identical on every path; irs_scan_tune times each candidate   */
/* on the batch (the choice cuBLAS makes inside the reference's dots).      */
/* ------------------------------------------------------------------------ */
typedef struct irs_scan irs_scan;
enum { IRS_SCAN_SPLIT = 0, IRS_SCAN_PAIR = 1, IRS_SCAN_FUSED = 2 };
typedef struct irs_scan_candidate {
  int32_t path;   /* IRS_SCAN_SPLIT, IRS_SCAN_PAIR or IRS_SCAN_FUSED */
  int32_t tile;   /* GEMM query-row tile width (256, 128, 64; 128 for the fused kernel) */
  uint64_t chunk; /* DB entries per chunk (a multiple of 32) */
} irs_scan_candidate;
typedef struct irs_scan_timing {
  irs_scan_candidate cand;
  double ms;        /* host wall time per pass, device synchronised */
  int32_t finalist; /* 0: the first round; 1: a finalist's mean over the interleaved rounds */
  int32_t reserved;
} irs_scan_timing;
/* The engines are the three parties' code and mask engines (party p at index
 * p); the scan keeps the handles, which must outlive it.  Starts configured
 * as IRS_SCAN_SPLIT with the engines' own tile, 65,536-entry chunks. */
int irs_scan_init(irs_device_manager* dm, irs_distance_comparator* dc, irs_circuits* c,
                  irs_sharedb* const code_engines[3], irs_sharedb* const mask_engines[3], size_t n_slots,
                  size_t db_len, uint32_t threshold_a, irs_scan** out);
int irs_scan_destroy(irs_scan* s);
/* The tuner's candidates for this batch shape: the two-launch path at every
 * tile width that divides the padded rows (64 only up to 768 rows), the
 * two-SM GEMM where the 256-row tile applies, the fused kernel where the rows
 * are a multiple of 128; chunks of 131,072 down to 8,192 entries capped at
 * the DB (the fused kernel on the three longest).  *n = the count; at most
 * cap are written. */
int irs_scan_candidates(irs_scan* s, irs_scan_candidate* out, size_t cap, size_t* n);
/* Packed uneven rows instead of plain slots: the candidates are for n_rows
 * padded query rows (0 = n_slots x 32) and, with use_segments != 0, every
 * pass evaluates the threshold through the comparator's stored segment table
 * (irs_dc_set_segments; irs_dc_compare_threshold_open_prepared, or the fused
 * kernel with use_segments), as BatchedEngine packs its variants. */
int irs_scan_set_rows(irs_scan* s, size_t n_rows, int use_segments);
/* Sets every engine's GEMM variant and tile for the path (set_pair /
 * set_tile) and the chunk length; the fused path allocates the comparator's
 * ring here, so configure it before any graph capture.  Clears the timing
 * events. */
int irs_scan_configure(irs_scan* s, int path, int tile, size_t chunk);
int irs_scan_current(irs_scan* s, irs_scan_candidate* cand);
/* One pass over the DB (the comparator is not reset) on `stream` (NULL =
 * party 0's stream); graph-capturable on party 0's stream when timing is
 * off and the configuration (and, for the fused path, its ring) was made
 * before the capture. */
int irs_scan_run(irs_scan* s, void* stream);
/* Per-chunk timing of the next max_passes passes (0 = off): CUDA events
 * before each chunk, after its GEMM (or fused launch) and after its
 * threshold launch, on the pass's stream.  irs_scan_timings waits for them
 * and writes per pass the GEMM, threshold and whole-pass milliseconds (*n =
 * passes recorded; reset != 0 starts over). */
int irs_scan_set_timing(irs_scan* s, size_t max_passes);
int irs_scan_timings(irs_scan* s, double* gemm_ms, double* threshold_ms, double* pass_ms, size_t cap, size_t* n,
                     int reset);
/* Times `passes` consecutive passes of every candidate (only those on path
 * `only_path` when >= 0) after a warm one (comparator reset before each),
 * re-times the `finalists` fastest interleaved for `rounds` rounds and
 * configures the best mean; `log` receives the first-round times, then each
 * finalist's mean (*n_log = the count; at most log_cap written). */
int irs_scan_tune(irs_scan* s, int passes, int finalists, int rounds, int only_path, irs_scan_candidate* chosen,
                  irs_scan_timing* log, size_t log_cap, size_t* n_log);
/* The engines back to the library's default GEMM (set_pair 0, set_tile 0). */
int irs_scan_restore(irs_scan* s);

/* ------------------------------------------------------------------------ */
/* CUDA graphs of a batch's device work (party 0's stream).  No counterpart */
/* in the reference, which launches every kernel through cudarc.            */
/* Between begin and end, the library keeps all launches on the capturing    */
/* stream (no cross-party event waits); calls that synchronise the host fail */
/* with the CUDA capture error.                                              */
/* ------------------------------------------------------------------------ */
typedef struct irs_graph irs_graph;
int irs_graph_begin_capture(irs_device_manager* dm);
int irs_graph_end_capture(irs_device_manager* dm, irs_graph** out);
int irs_graph_launch(irs_graph* g, void* stream);
int irs_graph_destroy(irs_graph* g);

#ifdef __cplusplus
}
#endif

#endif /* IRISB200_H */
