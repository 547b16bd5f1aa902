// C ABI of the B200 iris hot path (declarations and reference citations in
// include/irisb200.h).  Host-side object management: per-party streams and
// memory pools, device-resident share databases, query staging, and the
// launches of the limb GEMM, the fused threshold kernels and the result
// kernels.  No entry point aborts: every failure returns a status and sets
// the thread's last-error string.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <map>
#include <string>
#include <vector>

#include "../../include/irisb200.h"
#include "or_tree.h"
#include "common.cuh"
#include "fused_scan.h"
#include "gemm_limb.h"
#include "internal.h"
#include "prep.h"
#include "results.h"
#include "threshold.h"

using namespace irs;

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

#define CU(call)                                                                                     \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess) return fail(IRS_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                       __FILE__, __LINE__);                                          \
  } while (0)

#define CHECK(cond, code, ...) \
  do {                         \
    if (!(cond)) return fail((code), __VA_ARGS__); \
  } while (0)

size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

}  // namespace

struct irs_device_manager {
  int device = 0;
  int n_sms = 148;
  cudaStream_t streams[3] = {nullptr, nullptr, nullptr};
  cudaMemPool_t pools[3] = {nullptr, nullptr, nullptr};
  int* d_err = nullptr;
  uint64_t* d_batch = nullptr;  // device batch counter (irs_device_manager_set_batch_counter)
  bool capturing = false;  // a graph capture on streams[0] is open
  cudaEvent_t graph_done = nullptr;  // recorded after each graph launch
  bool host_sync = true;  // false: host-buffer calls return once enqueued (irs_device_manager_set_host_sync)
  // stage timers (irs_device_manager_set_timing): event pairs per label, resolved on read
  bool timing = false;
  struct Timer {
    const char* label;
    cudaEvent_t start, stop;
  };
  std::vector<Timer> timers;
  std::map<std::string, std::pair<double, long>> timer_totals;  // label -> (ms, launches)
  uint64_t stall_limit_ns = 0;  // armed by irs_device_manager_test_stall_next_dot (one shot)
};

// Brackets one stage launch on stream s with a pair of timing events when the
// device manager's stage timers are on (outside graph capture).
struct StageTimer {
  irs_device_manager* dm;
  cudaStream_t s;
  cudaEvent_t a = nullptr, b = nullptr;
  const char* label;
  StageTimer(irs_device_manager* d, cudaStream_t st, const char* l) : dm(d), s(st), label(l) {
    if (!dm->timing || dm->capturing) return;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
      cudaGetLastError();
      a = b = nullptr;
      return;
    }
    cudaEventRecord(a, s);
  }
  ~StageTimer() {
    if (!a) return;
    cudaEventRecord(b, s);
    dm->timers.push_back({label, a, b});
  }
};

struct irs_graph {
  irs_device_manager* dm = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

struct irs_sharedb {
  irs_device_manager* dm = nullptr;
  int peer = 0;
  size_t max_db = 0, query_length = 0, code_length = 0;
  ChaChaKey seed0{}, seed1{};
  bool remote = false;
  // device-resident DB limb planes [db_cap][K]
  uint8_t* db_lo = nullptr;
  uint8_t* db_hi = nullptr;
  size_t db_cap = 0, db_len = 0;
  // query limb planes [n_pad][K]
  uint8_t* q_lo = nullptr;
  uint8_t* q_hi = nullptr;
  uint16_t* q_stage = nullptr;  // u16 staging [n_pad][K]
  QuerySlot* d_slots = nullptr;
  size_t n_pad = 0;          // active padded query rows (result row stride)
  size_t n_cap = 0;          // query row capacity
  size_t rows_uploaded = 0;  // rows of the last upload
  int tile_override = 0;     // tile width requested by irs_sharedb_set_tile (0 = auto)
  bool pair = false;         // two-SM GEMM for the 256-row tile (irs_sharedb_set_pair)
  bool batch_from_device = false;
  bool have_query = false;
  // results [max_db][n_pad] u16 (entry-major)
  uint16_t* results = nullptr;
  size_t res_offset = 0, res_len = 0;
  uint64_t batch = 0;
  CUtensorMap tm_db_lo{}, tm_db_hi{}, tm_q_lo{}, tm_q_hi{};
  int block_n = 0;
  cudaEvent_t done = nullptr;  // recorded after the engine's last dot launch
};

struct irs_circuits {
  irs_device_manager* dm = nullptr;
  ChaChaKey keys[3]{};
  uint64_t batch = 0;
  bool batch_from_device = false;
};

struct irs_distance_comparator {
  irs_device_manager* dm = nullptr;
  size_t max_queries = 0, max_db = 0, stride_bits = 0, self_stride_bits = 0, match_cap = 0;
  uint32_t* bitmap = nullptr;       // [max_queries][stride_bits/32]
  uint32_t* self_bitmap = nullptr;  // [max_queries][self_stride_bits/32]
  uint32_t* match_list = nullptr;   // pairs
  uint32_t* counters = nullptr;     // [0] match count, [1] partial count
  uint32_t* partial = nullptr;      // [max_db] compaction output
  uint32_t* final_results = nullptr;  // [max_queries]
  uint32_t* match_counters = nullptr; // [max_queries]
  uint32_t* all_matches = nullptr;    // [max_queries][256]
  uint32_t* d_slot_valid = nullptr;
  uint32_t* d_slot_query = nullptr;
  uint32_t* d_take = nullptr;  // irs_dc_take_rows: row list [max_queries], counts [max_queries], ids [max_queries][256]
  // distance capture (irs_dc_enable_distance_capture): count, entry, row, code [3], mask [3]
  uint32_t* d_dist = nullptr;
  size_t dist_cap = 0;
  uint32_t* d_forced = nullptr;  // forced records: query [256], entry [256]
  uint32_t n_forced = 0;
  size_t slot_cap = 0;
  // segment table (irs_dc_set_segments)
  uint32_t* d_seg_start = nullptr;  // [slot_cap + 1]
  uint32_t* d_seg_query = nullptr;  // [seg_cap]
  uint32_t* d_seg_mask = nullptr;   // [seg_cap]
  size_t seg_cap = 0, n_seg_slots = 0;
  bool have_segments = false;
  // dot-share ring of the fused scan (irs_dc_scan_fused), allocated on first use
  uint16_t* ring = nullptr;
  size_t ring_bytes = 0;
};

namespace {

cudaStream_t party_stream(irs_device_manager* dm, int party, void* s) {
  return s ? static_cast<cudaStream_t>(s) : dm->streams[party];
}

int pool_alloc(irs_device_manager* dm, int party, size_t bytes, void** out) {
  *out = nullptr;
  if (!bytes) return IRS_OK;
  cudaError_t e = cudaMallocFromPoolAsync(out, bytes, dm->pools[party], dm->streams[party]);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(IRS_ERR_NOMEM, "device allocation of %zu bytes for party %d failed: %s", bytes, party,
                cudaGetErrorString(e));
  }
  e = cudaStreamSynchronize(dm->streams[party]);
  if (e != cudaSuccess) return fail(IRS_ERR_CUDA, "allocation sync: %s", cudaGetErrorString(e));
  return IRS_OK;
}

void pool_free(irs_device_manager* dm, int party, void* p) {
  if (p) cudaFreeAsync(p, dm->streams[party]);
}

int check_device_error(irs_device_manager* dm) {
  int code = 0;
  CU(cudaMemcpy(&code, dm->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (code) return fail(IRS_ERR_DEVICE, "kernel reported error code %d (bounded wait expired)", code);
  return IRS_OK;
}

ChaChaKey key_of(const uint32_t k[8]) {
  ChaChaKey r;
  for (int i = 0; i < 8; i++) r.k[i] = k[i];
  return r;
}

// Query tensor maps for the current tile width (the two-SM GEMM loads half of
// a query tile per CTA).
int rebuild_query_maps(irs_sharedb* db) {
  if (db->block_n <= 0) return IRS_OK;  // no valid tile width: dot reports it
  const uint32_t q_box = (uint32_t)(gemm_pair_applies(db->pair, db->block_n) ? db->block_n / 2 : db->block_n);
  if (make_tmap_u8(&db->tm_q_lo, db->q_lo, db->n_cap, db->code_length, q_box) ||
      make_tmap_u8(&db->tm_q_hi, db->q_hi, db->n_cap, db->code_length, q_box))
    return fail(IRS_ERR_CUDA, "tensor map for the query planes failed");
  return IRS_OK;
}

// Sets the active padded row count and tile width for `rows` query rows.
// Padded query rows for `rows` real rows: a multiple of 64, raised to a
// multiple of 128 (up to 768 rows) or 256 (above) when the query capacity
// allows, so that the GEMM runs the tile gemm_block_n_for picks for that row
// count instead of falling back to the 64-row tile (1600 rows on the 64-row
// tile take about twice as long as 1792 rows on the 256-row tile).  The extra
// rows are zero and no comparison reads them.
static size_t padded_query_rows(size_t rows, size_t n_cap) {
  const size_t n64 = round_up(rows ? rows : 1, 64);
  const size_t wide = n64 <= 64 ? n64 : (n64 <= 768 ? round_up(n64, 128) : round_up(n64, 256));
  return wide <= n_cap ? wide : n64;
}

int set_active_rows(irs_sharedb* db, size_t rows) {
  const size_t n = padded_query_rows(rows, db->n_cap);
  if (n > db->n_cap) return fail(IRS_ERR_INVALID, "%zu rows exceed the query capacity %zu", rows, db->n_cap);
  int bn = gemm_block_n_for((uint32_t)n);
  if (db->tile_override && n % (size_t)db->tile_override == 0) bn = db->tile_override;
  const bool rebuild = bn != db->block_n;
  db->n_pad = n;
  db->block_n = bn;
  db->rows_uploaded = rows;
  return rebuild ? rebuild_query_maps(db) : IRS_OK;
}

}  // namespace

extern "C" {

const char* irs_last_error(void) { return g_err; }

const char* irs_version(void) { return "irisb200 0.1 (sm_100a, tcgen05 i8 limb GEMM, fused 3-party threshold)"; }

// ---------------------------------------------------------------------------
// Device manager
// ---------------------------------------------------------------------------
int irs_device_manager_init(int device, irs_device_manager** out) {
  CHECK(out, IRS_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int n = 0;
  CU(cudaGetDeviceCount(&n));
  CHECK(device >= 0 && device < n, IRS_ERR_INVALID, "device %d out of range (%d devices)", device, n);
  CU(cudaSetDevice(device));
  cudaDeviceProp prop;
  CU(cudaGetDeviceProperties(&prop, device));
  CHECK(prop.major == 10 && prop.minor == 0, IRS_ERR_INVALID,
        "device %d is sm_%d%d; this library is built for sm_100a (B200)", device, prop.major, prop.minor);
  auto* dm = new (std::nothrow) irs_device_manager();
  CHECK(dm, IRS_ERR_NOMEM, "host allocation failed");
  dm->device = device;
  dm->n_sms = prop.multiProcessorCount;
  for (int p = 0; p < 3; p++) {
    CU(cudaStreamCreateWithFlags(&dm->streams[p], cudaStreamNonBlocking));
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    CU(cudaMemPoolCreate(&dm->pools[p], &props));
    uint64_t threshold = UINT64_MAX;
    CU(cudaMemPoolSetAttribute(dm->pools[p], cudaMemPoolAttrReleaseThreshold, &threshold));
  }
  CU(cudaMalloc(&dm->d_err, sizeof(int)));
  CU(cudaMemset(dm->d_err, 0, sizeof(int)));
  CU(cudaMalloc(&dm->d_batch, sizeof(uint64_t)));
  CU(cudaMemset(dm->d_batch, 0, sizeof(uint64_t)));
  CU(cudaEventCreateWithFlags(&dm->graph_done, cudaEventDisableTiming));
  *out = dm;
  return IRS_OK;
}

int irs_device_manager_destroy(irs_device_manager* dm) {
  if (!dm) return IRS_OK;
  cudaSetDevice(dm->device);
  for (int p = 0; p < 3; p++) if (dm->streams[p]) cudaStreamSynchronize(dm->streams[p]);
  cudaFree(dm->d_err);
  cudaFree(dm->d_batch);
  if (dm->graph_done) cudaEventDestroy(dm->graph_done);
  for (auto& t : dm->timers) {
    cudaEventDestroy(t.start);
    cudaEventDestroy(t.stop);
  }
  for (int p = 0; p < 3; p++) {
    if (dm->streams[p]) cudaStreamDestroy(dm->streams[p]);
    if (dm->pools[p]) cudaMemPoolDestroy(dm->pools[p]);
  }
  delete dm;
  return IRS_OK;
}

int irs_device_manager_stream(irs_device_manager* dm, int party, void** stream) {
  CHECK(dm && stream && party >= 0 && party < 3, IRS_ERR_INVALID, "bad arguments");
  *stream = dm->streams[party];
  return IRS_OK;
}

int irs_device_manager_synchronize(irs_device_manager* dm) {
  CHECK(dm, IRS_ERR_INVALID, "dm is NULL");
  for (int p = 0; p < 3; p++) CU(cudaStreamSynchronize(dm->streams[p]));
  return check_device_error(dm);
}

int irs_device_manager_error(irs_device_manager* dm, int* code) {
  CHECK(dm && code, IRS_ERR_INVALID, "bad arguments");
  CU(cudaMemcpy(code, dm->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  return IRS_OK;
}

int irs_device_manager_clear_error(irs_device_manager* dm) {
  CHECK(dm, IRS_ERR_INVALID, "dm is NULL");
  CU(cudaMemset(dm->d_err, 0, sizeof(int)));
  return IRS_OK;
}

int irs_device_manager_test_stall_next_dot(irs_device_manager* dm, uint64_t wait_limit_ns) {
  CHECK(dm, IRS_ERR_INVALID, "dm is NULL");
  CHECK(wait_limit_ns >= 1000 && wait_limit_ns <= 10000000000ull, IRS_ERR_INVALID,
        "wait limit %llu ns outside 1 us .. 10 s", (unsigned long long)wait_limit_ns);
  CHECK(!dm->capturing, IRS_ERR_STATE, "arm the stall outside a graph capture");
  dm->stall_limit_ns = wait_limit_ns;
  return IRS_OK;
}

int irs_device_manager_set_batch_counter(irs_device_manager* dm, uint64_t batch_id, void* stream) {
  CHECK(dm, IRS_ERR_INVALID, "dm is NULL");
  CHECK(batch_id < (1ull << 24), IRS_ERR_INVALID, "batch id must be below 2^24");
  CHECK(!dm->capturing, IRS_ERR_STATE, "set the batch counter outside a graph capture");
  static thread_local uint64_t staged;  // pageable source; the copy is synchronised below
  staged = batch_id;
  cudaStream_t s = party_stream(dm, 0, stream);
  CU(cudaMemcpyAsync(dm->d_batch, &staged, sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  CU(cudaStreamSynchronize(s));
  return IRS_OK;
}

__global__ void advance_batch_counter_kernel(uint64_t* b) { *b = *b % ((1ull << 24) - 1) + 1; }

int irs_device_manager_set_timing(irs_device_manager* dm, int on) {
  CHECK(dm, IRS_ERR_INVALID, "dm is NULL");
  dm->timing = on != 0;
  return IRS_OK;
}

int irs_device_manager_timings(irs_device_manager* dm, char* buf, size_t cap, int reset) {
  CHECK(dm && buf && cap > 0, IRS_ERR_INVALID, "bad arguments");
  CU(cudaSetDevice(dm->device));
  for (auto& t : dm->timers) {
    float ms = 0.f;
    CU(cudaEventSynchronize(t.stop));
    CU(cudaEventElapsedTime(&ms, t.start, t.stop));
    auto& tot = dm->timer_totals[t.label];
    tot.first += ms;
    tot.second += 1;
    cudaEventDestroy(t.start);
    cudaEventDestroy(t.stop);
  }
  dm->timers.clear();
  std::string out;
  char line[160];
  for (auto& kv : dm->timer_totals) {
    snprintf(line, sizeof line, "%s%s=%.6f/%ld", out.empty() ? "" : ";", kv.first.c_str(), kv.second.first,
             kv.second.second);
    out += line;
  }
  CHECK(out.size() + 1 <= cap, IRS_ERR_OVERFLOW, "timings need %zu bytes", out.size() + 1);
  memcpy(buf, out.c_str(), out.size() + 1);
  if (reset) dm->timer_totals.clear();
  return IRS_OK;
}

int irs_device_manager_get_batch_counter(irs_device_manager* dm, uint64_t* batch_id) {
  CHECK(dm && batch_id, IRS_ERR_INVALID, "bad arguments");
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[0];
  CU(cudaMemcpyAsync(batch_id, dm->d_batch, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  return IRS_OK;
}

int irs_device_manager_advance_batch_counter(irs_device_manager* dm, void* stream) {
  CHECK(dm, IRS_ERR_INVALID, "dm is NULL");
  CU(cudaSetDevice(dm->device));
  advance_batch_counter_kernel<<<1, 1, 0, party_stream(dm, 0, stream)>>>(dm->d_batch);
  CU(cudaGetLastError());
  return IRS_OK;
}

int irs_sharedb_use_batch_counter(irs_sharedb* db, int on) {
  CHECK(db, IRS_ERR_INVALID, "db is NULL");
  db->batch_from_device = on != 0;
  return IRS_OK;
}

int irs_circuits_use_batch_counter(irs_circuits* c, int on) {
  CHECK(c, IRS_ERR_INVALID, "c is NULL");
  c->batch_from_device = on != 0;
  return IRS_OK;
}

int irs_device_manager_set_host_sync(irs_device_manager* dm, int on) {
  CHECK(dm, IRS_ERR_INVALID, "dm is NULL");
  dm->host_sync = on != 0;
  return IRS_OK;
}

int irs_event_create(void** ev) {
  CHECK(ev, IRS_ERR_INVALID, "ev is NULL");
  cudaEvent_t e = nullptr;
  CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  *ev = e;
  return IRS_OK;
}

int irs_event_record(void* ev, void* stream) {
  CHECK(ev, IRS_ERR_INVALID, "ev is NULL");
  CU(cudaEventRecord(static_cast<cudaEvent_t>(ev), static_cast<cudaStream_t>(stream)));
  return IRS_OK;
}

int irs_event_synchronize(void* ev) {
  CHECK(ev, IRS_ERR_INVALID, "ev is NULL");
  CU(cudaEventSynchronize(static_cast<cudaEvent_t>(ev)));
  return IRS_OK;
}

int irs_event_query(void* ev, int* done) {
  CHECK(ev && done, IRS_ERR_INVALID, "bad arguments");
  const cudaError_t e = cudaEventQuery(static_cast<cudaEvent_t>(ev));
  if (e == cudaErrorNotReady) {
    *done = 0;
    return IRS_OK;
  }
  CU(e);
  *done = 1;
  return IRS_OK;
}

int irs_event_destroy(void* ev) {
  if (ev) cudaEventDestroy(static_cast<cudaEvent_t>(ev));
  return IRS_OK;
}

int irs_device_manager_mem_info(irs_device_manager* dm, size_t* free_bytes, size_t* total_bytes) {
  CHECK(dm && free_bytes && total_bytes, IRS_ERR_INVALID, "bad arguments");
  CU(cudaSetDevice(dm->device));
  CU(cudaMemGetInfo(free_bytes, total_bytes));
  return IRS_OK;
}

int irs_device_manager_sm_count(irs_device_manager* dm, int* n) {
  CHECK(dm && n, IRS_ERR_INVALID, "bad arguments");
  *n = dm->n_sms;
  return IRS_OK;
}

int irs_device_alloc(irs_device_manager* dm, size_t bytes, void** ptr) {
  CHECK(dm && ptr, IRS_ERR_INVALID, "bad arguments");
  cudaError_t e = cudaMalloc(ptr, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(IRS_ERR_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  }
  return IRS_OK;
}

int irs_host_alloc_pinned(size_t bytes, void** ptr) {
  CHECK(ptr, IRS_ERR_INVALID, "ptr is NULL");
  cudaError_t e = cudaMallocHost(ptr, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(IRS_ERR_NOMEM, "cudaMallocHost(%zu): %s", bytes, cudaGetErrorString(e));
  }
  return IRS_OK;
}

int irs_host_free_pinned(void* ptr) {
  if (ptr) CU(cudaFreeHost(ptr));
  return IRS_OK;
}

int irs_device_free(irs_device_manager* dm, void* ptr) {
  (void)dm;
  if (ptr) CU(cudaFree(ptr));
  return IRS_OK;
}

int irs_copy_h2d(void* dst, const void* src, size_t bytes, void* stream) {
  CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream)));
  return IRS_OK;
}

int irs_copy_d2h(void* dst, const void* src, size_t bytes, void* stream) {
  CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)));
  return IRS_OK;
}

int irs_stream_synchronize(void* stream) {
  CU(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  return IRS_OK;
}

// ---------------------------------------------------------------------------
// ShareDB
// ---------------------------------------------------------------------------
int irs_sharedb_init(irs_device_manager* dm, int peer_id, size_t max_db_length, size_t query_length,
                     size_t code_length, const uint32_t seed0[8], const uint32_t seed1[8], int is_remote,
                     irs_sharedb** out) {
  CHECK(dm && out && seed0 && seed1, IRS_ERR_INVALID, "bad arguments");
  *out = nullptr;
  CHECK(peer_id >= 0 && peer_id < 3, IRS_ERR_INVALID, "peer_id %d not in 0..2", peer_id);
  CHECK(code_length > 0 && code_length % 128 == 0, IRS_ERR_INVALID, "code_length %zu must be a multiple of 128",
        code_length);
  CHECK(query_length > 0 && query_length <= 65536, IRS_ERR_INVALID, "query_length %zu out of range", query_length);
  CHECK(max_db_length > 0 && max_db_length < (1ull << 31), IRS_ERR_INVALID, "max_db_length %zu out of range",
        max_db_length);
  CU(cudaSetDevice(dm->device));
  auto* db = new (std::nothrow) irs_sharedb();
  CHECK(db, IRS_ERR_NOMEM, "host allocation failed");
  db->dm = dm;
  db->peer = peer_id;
  db->max_db = max_db_length;
  db->query_length = query_length;
  db->code_length = code_length;
  db->seed0 = key_of(seed0);
  db->seed1 = key_of(seed1);
  db->remote = is_remote != 0;
  db->n_cap = round_up(query_length, 64);
  db->n_pad = db->n_cap;
  db->block_n = gemm_block_n_for((uint32_t)db->n_pad);
  if (cudaEventCreateWithFlags(&db->done, cudaEventDisableTiming) != cudaSuccess) {
    delete db;
    return fail(IRS_ERR_CUDA, "event creation failed");
  }
  int rc;
  void* p;
  if ((rc = pool_alloc(dm, peer_id, db->n_cap * code_length, &p))) { irs_sharedb_destroy(db); return rc; }
  db->q_lo = (uint8_t*)p;
  if ((rc = pool_alloc(dm, peer_id, db->n_cap * code_length, &p))) { irs_sharedb_destroy(db); return rc; }
  db->q_hi = (uint8_t*)p;
  if ((rc = pool_alloc(dm, peer_id, db->n_cap * code_length * 2, &p))) { irs_sharedb_destroy(db); return rc; }
  db->q_stage = (uint16_t*)p;
  if ((rc = pool_alloc(dm, peer_id, (db->n_cap / kSlotRows) * sizeof(QuerySlot), &p))) { irs_sharedb_destroy(db); return rc; }
  db->d_slots = (QuerySlot*)p;
  if ((rc = pool_alloc(dm, peer_id, max_db_length * db->n_cap * 2, &p))) { irs_sharedb_destroy(db); return rc; }
  db->results = (uint16_t*)p;
  if ((rc = rebuild_query_maps(db))) {
    irs_sharedb_destroy(db);
    return rc;
  }
  *out = db;
  return IRS_OK;
}

int irs_sharedb_destroy(irs_sharedb* db) {
  if (!db) return IRS_OK;
  irs_device_manager* dm = db->dm;
  cudaSetDevice(dm->device);
  pool_free(dm, db->peer, db->db_lo);
  pool_free(dm, db->peer, db->db_hi);
  pool_free(dm, db->peer, db->q_lo);
  pool_free(dm, db->peer, db->q_hi);
  pool_free(dm, db->peer, db->q_stage);
  pool_free(dm, db->peer, db->d_slots);
  pool_free(dm, db->peer, db->results);
  cudaStreamSynchronize(dm->streams[db->peer]);
  if (db->done) cudaEventDestroy(db->done);
  delete db;
  return IRS_OK;
}

int irs_sharedb_alloc_db(irs_sharedb* db, size_t max_db_length) {
  CHECK(db, IRS_ERR_INVALID, "db is NULL");
  CHECK(max_db_length > 0 && max_db_length < (1ull << 31), IRS_ERR_INVALID, "max_db_length %zu out of range",
        max_db_length);
  irs_device_manager* dm = db->dm;
  CU(cudaSetDevice(dm->device));
  pool_free(dm, db->peer, db->db_lo);
  pool_free(dm, db->peer, db->db_hi);
  db->db_lo = db->db_hi = nullptr;
  const size_t cap = round_up(max_db_length, 128);
  void* p;
  int rc;
  if ((rc = pool_alloc(dm, db->peer, cap * db->code_length, &p))) return rc;
  db->db_lo = (uint8_t*)p;
  if ((rc = pool_alloc(dm, db->peer, cap * db->code_length, &p))) return rc;
  db->db_hi = (uint8_t*)p;
  CU(cudaMemsetAsync(db->db_lo, 0, cap * db->code_length, dm->streams[db->peer]));
  CU(cudaMemsetAsync(db->db_hi, 0, cap * db->code_length, dm->streams[db->peer]));
  db->db_cap = cap;
  db->db_len = 0;
  if (make_tmap_u8(&db->tm_db_lo, db->db_lo, cap, db->code_length, 128) ||
      make_tmap_u8(&db->tm_db_hi, db->db_hi, cap, db->code_length, 128))
    return fail(IRS_ERR_CUDA, "tensor map for the DB planes failed");
  CU(cudaStreamSynchronize(dm->streams[db->peer]));
  return IRS_OK;
}

int irs_sharedb_load_records(irs_sharedb* db, size_t first, size_t n, const uint16_t* records) {
  CHECK(db && (records || !n), IRS_ERR_INVALID, "bad arguments");
  CHECK(db->db_lo, IRS_ERR_STATE, "alloc_db not called");
  CHECK(first + n <= db->db_cap, IRS_ERR_INVALID, "records %zu..%zu exceed the DB capacity %zu", first, first + n,
        db->db_cap);
  irs_device_manager* dm = db->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[db->peer];
  const size_t K = db->code_length;
  const size_t per = std::max<size_t>(1, db->n_cap);  // records per pass through the query staging buffer
  for (size_t done = 0; done < n;) {
    const size_t c = std::min(per, n - done);
    CU(cudaMemcpyAsync(db->q_stage, records + done * K, c * K * 2, cudaMemcpyHostToDevice, s));
    CU(launch_split_limbs(db->q_stage, db->db_lo + (first + done) * K, db->db_hi + (first + done) * K, c * K, s));
    CU(cudaStreamSynchronize(s));
    done += c;
  }
  db->db_len = std::max(db->db_len, first + n);
  return IRS_OK;
}

int irs_sharedb_load_records_i8(irs_sharedb* db, size_t first, size_t n, const uint8_t* limb0, const uint8_t* limb1) {
  CHECK(db && ((limb0 && limb1) || !n), IRS_ERR_INVALID, "bad arguments");
  CHECK(db->db_lo, IRS_ERR_STATE, "alloc_db not called");
  CHECK(first + n <= db->db_cap, IRS_ERR_INVALID, "records exceed the DB capacity");
  irs_device_manager* dm = db->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[db->peer];
  const size_t K = db->code_length;
  CU(cudaMemcpyAsync(db->db_lo + first * K, limb0, n * K, cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(db->db_hi + first * K, limb1, n * K, cudaMemcpyHostToDevice, s));
  CU(launch_xor80(db->db_lo + first * K, n * K, s));
  CU(launch_xor80(db->db_hi + first * K, n * K, s));
  CU(cudaStreamSynchronize(s));
  db->db_len = std::max(db->db_len, first + n);
  return IRS_OK;
}

int irs_sharedb_fetch_records(irs_sharedb* db, size_t first, size_t n, uint16_t* records) {
  CHECK(db && (records || !n), IRS_ERR_INVALID, "bad arguments");
  CHECK(db->db_lo, IRS_ERR_STATE, "alloc_db not called");
  CHECK(first + n <= db->db_cap, IRS_ERR_INVALID, "records exceed the DB capacity");
  irs_device_manager* dm = db->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[db->peer];
  const size_t K = db->code_length;
  std::vector<uint8_t> lo(n * K), hi(n * K);
  CU(cudaMemcpyAsync(lo.data(), db->db_lo + first * K, n * K, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(hi.data(), db->db_hi + first * K, n * K, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  for (size_t i = 0; i < n * K; i++) records[i] = (uint16_t)(lo[i] | (hi[i] << 8));
  return IRS_OK;
}

int irs_sharedb_set_db_len(irs_sharedb* db, size_t len) {
  CHECK(db, IRS_ERR_INVALID, "db is NULL");
  CHECK(len <= db->db_cap, IRS_ERR_INVALID, "len %zu exceeds capacity %zu", len, db->db_cap);
  db->db_len = len;
  return IRS_OK;
}

int irs_sharedb_db_len(irs_sharedb* db, size_t* len) {
  CHECK(db && len, IRS_ERR_INVALID, "bad arguments");
  *len = db->db_len;
  return IRS_OK;
}

int irs_sharedb_synth_db(irs_sharedb* const code_engines[3], irs_sharedb* const mask_engines[3], uint64_t seed,
                         size_t first, size_t n) {
  SynthOut o;
  for (int p = 0; p < 3; p++) {
    irs_sharedb* c = code_engines[p];
    irs_sharedb* m = mask_engines[p];
    CHECK(c && m && c->db_lo && m->db_lo, IRS_ERR_STATE, "engines of party %d need alloc_db", p);
    CHECK(c->code_length == (size_t)kIrisCodeLength && m->code_length == (size_t)kMaskCodeLength, IRS_ERR_INVALID,
          "synthetic DB needs code_length 12800 / 6400 engines");
    CHECK(first + n <= c->db_cap && first + n <= m->db_cap, IRS_ERR_INVALID, "records exceed the DB capacity");
    o.code_lo[p] = c->db_lo; o.code_hi[p] = c->db_hi;
    o.mask_lo[p] = m->db_lo; o.mask_hi[p] = m->db_hi;
  }
  irs_device_manager* dm = code_engines[0]->dm;
  CU(cudaSetDevice(dm->device));
  for (int p = 0; p < 3; p++) {
    CU(cudaStreamSynchronize(dm->streams[p]));
  }
  const size_t step = 1u << 20;
  for (size_t done = 0; done < n; done += step) {
    const uint32_t c = (uint32_t)std::min(step, n - done);
    CU(launch_synth_db(seed, (uint32_t)(first + done), c, o, dm->streams[0]));
  }
  CU(cudaStreamSynchronize(dm->streams[0]));
  for (int p = 0; p < 3; p++) {
    code_engines[p]->db_len = std::max(code_engines[p]->db_len, first + n);
    mask_engines[p]->db_len = std::max(mask_engines[p]->db_len, first + n);
  }
  return IRS_OK;
}

// Orders a write to an engine's query rows or records on stream s after the
// last GEMM that read them (a direct launch, or a graph launch).
static cudaError_t wait_last_dot(irs_sharedb* db, cudaStream_t s) {
  cudaError_t e = cudaStreamWaitEvent(s, db->done, 0);
  if (e != cudaSuccess) return e;
  return cudaStreamWaitEvent(s, db->dm->graph_done, 0);
}

int irs_sharedb_fill_random(irs_sharedb* db, uint64_t seed, size_t n) {
  CHECK(db && db->db_lo, IRS_ERR_STATE, "alloc_db not called");
  CHECK(n <= db->db_cap, IRS_ERR_INVALID, "%zu records exceed the DB capacity %zu", n, db->db_cap);
  CHECK((n * db->code_length) % 8 == 0, IRS_ERR_INVALID, "records x code_length must be a multiple of 8");
  irs_device_manager* dm = db->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[db->peer];
  CU(wait_last_dot(db, s));
  CU(launch_fill_random(db->db_lo, n * db->code_length, seed, s));
  CU(launch_fill_random(db->db_hi, n * db->code_length, seed ^ 0x5A5A5A5A5A5A5A5Aull, s));
  CU(cudaStreamSynchronize(s));
  db->db_len = std::max(db->db_len, n);
  return IRS_OK;
}

int irs_device_fill_random(void* ptr, size_t bytes, uint64_t seed, void* stream) {
  CHECK(ptr && bytes % 8 == 0 && reinterpret_cast<uintptr_t>(ptr) % 8 == 0, IRS_ERR_INVALID,
        "8-byte aligned pointer and a multiple of 8 bytes needed");
  CU(launch_fill_random(ptr, bytes, seed, static_cast<cudaStream_t>(stream)));
  return IRS_OK;
}

int irs_sharedb_query_upload(irs_sharedb* db, const uint16_t* rows, size_t n_rows) {
  CHECK(db && (rows || !n_rows), IRS_ERR_INVALID, "bad arguments");
  int rc = set_active_rows(db, n_rows);
  if (rc) return rc;
  irs_device_manager* dm = db->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[db->peer];
  CU(wait_last_dot(db, s));  // the last GEMM has read the old limb planes
  const size_t K = db->code_length;
  CU(cudaMemsetAsync(db->q_stage, 0, db->n_pad * K * 2, s));
  if (n_rows) CU(cudaMemcpyAsync(db->q_stage, rows, n_rows * K * 2, cudaMemcpyHostToDevice, s));
  CU(launch_split_limbs(db->q_stage, db->q_lo, db->q_hi, db->n_pad * K, s));
  db->have_query = true;
  return IRS_OK;
}

int irs_sharedb_query_upload_slots(irs_sharedb* db, const uint16_t* base, size_t n_base, const irs_query_slot* slots,
                                   size_t n_slots) {
  CHECK(db && base && slots && n_base > 0, IRS_ERR_INVALID, "bad arguments");
  CHECK(n_slots * kSlotRows <= db->n_cap, IRS_ERR_INVALID, "%zu slots exceed the query capacity %zu", n_slots,
        db->n_cap);
  CHECK(n_base <= db->n_cap, IRS_ERR_INVALID, "too many base queries");
  CHECK(db->code_length % kRowLen == 0, IRS_ERR_INVALID, "rotations need code_length a multiple of 800");
  for (size_t i = 0; i < n_slots; i++) {
    CHECK(slots[i].src < n_base && slots[i].n_rot <= (uint32_t)kRotations &&
              slots[i].rot_lo + slots[i].n_rot <= (uint32_t)kRotations,
          IRS_ERR_INVALID, "slot %zu is invalid", i);
  }
  int rc = set_active_rows(db, n_slots * kSlotRows);
  if (rc) return rc;
  irs_device_manager* dm = db->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[db->peer];
  CU(wait_last_dot(db, s));
  const size_t K = db->code_length;
  CU(cudaMemcpyAsync(db->q_stage, base, n_base * K * 2, cudaMemcpyHostToDevice, s));
  static_assert(sizeof(QuerySlot) == sizeof(irs_query_slot), "slot layout");
  CU(cudaMemcpyAsync(db->d_slots, slots, n_slots * sizeof(QuerySlot), cudaMemcpyHostToDevice, s));
  CU(launch_expand_slots(db->q_stage, (uint32_t)K, db->d_slots, (uint32_t)n_slots, (uint32_t)db->n_pad, db->q_lo,
                         db->q_hi, s));
  CU(cudaStreamSynchronize(s));  // slots / base are caller-owned host memory
  db->have_query = true;
  return IRS_OK;
}

int irs_sharedb_query_upload_rows(irs_sharedb* db, const uint16_t* base, size_t n_base, const uint32_t* row_desc,
                                  size_t n_rows) {
  CHECK(db && base && row_desc && n_base > 0, IRS_ERR_INVALID, "bad arguments");
  CHECK(db->code_length % kRowLen == 0, IRS_ERR_INVALID, "rotations need code_length a multiple of 800");
  const size_t K = db->code_length;
  // staging: base queries, then the row table after them
  const size_t base_bytes = n_base * K * 2, table_bytes = n_rows * 4;
  CHECK(base_bytes + table_bytes + 16 <= db->n_cap * K * 2, IRS_ERR_INVALID, "too many base queries for the staging");
  for (size_t r = 0; r < n_rows; r++)
    CHECK(row_desc[r] == 0xFFFFFFFFu || ((row_desc[r] >> 8) < n_base && (row_desc[r] & 0x7Fu) < (uint32_t)kRotations),
          IRS_ERR_INVALID, "row %zu descriptor 0x%x is invalid", r, row_desc[r]);
  int rc = set_active_rows(db, n_rows);
  if (rc) return rc;
  irs_device_manager* dm = db->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[db->peer];
  CU(wait_last_dot(db, s));
  uint8_t* stage = reinterpret_cast<uint8_t*>(db->q_stage);
  const size_t table_off = (base_bytes + 15) / 16 * 16;
  CU(cudaMemcpyAsync(stage, base, base_bytes, cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(stage + table_off, row_desc, table_bytes, cudaMemcpyHostToDevice, s));
  CU(launch_expand_rows(db->q_stage, (uint32_t)K, reinterpret_cast<const uint32_t*>(stage + table_off), (uint32_t)n_rows,
                        (uint32_t)db->n_pad, db->q_lo, db->q_hi, s));
  if (dm->host_sync) CU(cudaStreamSynchronize(s));  // base / row_desc are caller-owned host memory
  db->have_query = true;
  return IRS_OK;
}

int irs_sharedb_query_put_base(irs_sharedb* db, size_t first, size_t n, const uint16_t* base) {
  CHECK(db && (base || !n), IRS_ERR_INVALID, "bad arguments");
  const size_t K = db->code_length;
  CHECK((first + n) * K * 2 + db->n_cap * 4 + 16 <= db->n_cap * K * 2, IRS_ERR_INVALID,
        "base queries [%zu, %zu) exceed the resident pool", first, first + n);
  irs_device_manager* dm = db->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[db->peer];
  if (n) {
    CU(cudaMemcpyAsync(db->q_stage + first * K, base, n * K * 2, cudaMemcpyHostToDevice, s));
    if (dm->host_sync) CU(cudaStreamSynchronize(s));  // caller-owned host memory
  }
  return IRS_OK;
}

int irs_sharedb_query_expand_rows(irs_sharedb* db, size_t n_base, const uint32_t* row_desc, size_t n_rows) {
  CHECK(db && row_desc && n_base > 0, IRS_ERR_INVALID, "bad arguments");
  CHECK(db->code_length % kRowLen == 0, IRS_ERR_INVALID, "rotations need code_length a multiple of 800");
  const size_t K = db->code_length;
  const size_t base_bytes = n_base * K * 2, table_bytes = n_rows * 4;
  CHECK(base_bytes + table_bytes + 16 <= db->n_cap * K * 2, IRS_ERR_INVALID, "pool and row table exceed the staging");
  for (size_t r = 0; r < n_rows; r++)
    CHECK(row_desc[r] == 0xFFFFFFFFu || ((row_desc[r] >> 8) < n_base && (row_desc[r] & 0x7Fu) < (uint32_t)kRotations),
          IRS_ERR_INVALID, "row %zu descriptor 0x%x is invalid", r, row_desc[r]);
  int rc = set_active_rows(db, n_rows);
  if (rc) return rc;
  irs_device_manager* dm = db->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[db->peer];
  CU(wait_last_dot(db, s));
  uint8_t* stage = reinterpret_cast<uint8_t*>(db->q_stage);
  const size_t table_off = (base_bytes + 15) / 16 * 16;
  CU(cudaMemcpyAsync(stage + table_off, row_desc, table_bytes, cudaMemcpyHostToDevice, s));
  CU(launch_expand_rows(db->q_stage, (uint32_t)K, reinterpret_cast<const uint32_t*>(stage + table_off), (uint32_t)n_rows,
                        (uint32_t)db->n_pad, db->q_lo, db->q_hi, s));
  if (dm->host_sync) CU(cudaStreamSynchronize(s));  // row_desc is caller-owned host memory
  db->have_query = true;
  return IRS_OK;
}

int irs_sharedb_gather_records(irs_sharedb* dst, irs_sharedb* src, const uint32_t* ids, size_t n) {
  CHECK(dst && src && (ids || !n), IRS_ERR_INVALID, "bad arguments");
  CHECK(dst->dm == src->dm && dst->peer == src->peer && dst->code_length == src->code_length, IRS_ERR_INVALID,
        "gather needs engines of the same party and code length");
  CHECK(dst->db_lo && src->db_lo, IRS_ERR_STATE, "alloc_db not called");
  CHECK(n <= dst->db_cap, IRS_ERR_INVALID, "%zu records exceed the destination capacity %zu", n, dst->db_cap);
  for (size_t k = 0; k < n; k++)
    CHECK(ids[k] < src->db_cap, IRS_ERR_INVALID, "record id %u out of range", ids[k]);
  irs_device_manager* dm = dst->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[dst->peer];
  CU(wait_last_dot(dst, s));  // the last GEMM over dst's records has finished
  const size_t K = dst->code_length;
  CHECK(n * 4 <= dst->n_cap * K * 2, IRS_ERR_INVALID, "too many records for one gather");
  // Staging reuse: the gather runs before the next query upload of `dst`.
  CU(cudaMemcpyAsync(dst->q_stage, ids, n * 4, cudaMemcpyHostToDevice, s));
  CU(launch_gather_rows(src->db_lo, src->db_hi, reinterpret_cast<const uint32_t*>(dst->q_stage), (uint32_t)n,
                        (uint32_t)K, dst->db_lo, dst->db_hi, s));
  if (dm->host_sync) CU(cudaStreamSynchronize(s));  // ids is caller-owned host memory
  dst->db_len = n;
  return IRS_OK;
}

int irs_sharedb_set_tile(irs_sharedb* db, int block_n) {
  CHECK(db, IRS_ERR_INVALID, "db is NULL");
  CHECK(block_n == 0 || block_n == 64 || block_n == 128 || block_n == 256, IRS_ERR_INVALID,
        "tile width %d is not 0, 64, 128 or 256", block_n);
  db->tile_override = block_n;
  if (db->have_query) return set_active_rows(db, db->rows_uploaded);
  return IRS_OK;
}

int irs_sharedb_set_pair(irs_sharedb* db, int on) {
  CHECK(db, IRS_ERR_INVALID, "db is NULL");
  const bool rebuild = db->pair != (on != 0) && db->block_n == 256;
  db->pair = on != 0;
  return rebuild ? rebuild_query_maps(db) : IRS_OK;
}

int irs_sharedb_set_batch(irs_sharedb* db, uint64_t batch_id) {
  CHECK(db, IRS_ERR_INVALID, "db is NULL");
  CHECK(batch_id < (1ull << 24), IRS_ERR_INVALID, "batch id must be below 2^24");
  db->batch = batch_id;
  return IRS_OK;
}

static int fill_problem(irs_sharedb* db, uint16_t mult, size_t offset, size_t len, GemmProblem& pr) {
  CHECK(db->db_lo, IRS_ERR_STATE, "alloc_db not called");
  CHECK(db->have_query, IRS_ERR_STATE, "no query uploaded");
  CHECK(offset % 32 == 0, IRS_ERR_INVALID, "offset %zu must be a multiple of 32", offset);
  CHECK(offset + len <= db->db_cap && len <= db->max_db, IRS_ERR_INVALID, "entries %zu..%zu out of range", offset,
        offset + len);
  CHECK(db->block_n > 0, IRS_ERR_INVALID, "padded query length %zu has no valid tile width", db->n_pad);
  memset(&pr, 0, sizeof pr);
  pr.tm_a_lo = db->tm_db_lo;
  pr.tm_a_hi = db->tm_db_hi;
  pr.tm_b_lo = db->tm_q_lo;
  pr.tm_b_hi = db->tm_q_hi;
  pr.out = db->results;
  pr.m0 = (uint32_t)offset;
  pr.m_len = (uint32_t)len;
  pr.n_pad = (uint32_t)db->n_pad;
  pr.k_iters = (uint32_t)(db->code_length / 128);
  pr.mult = mult;
  pr.mask_on = db->remote ? 1u : 0u;
  pr.key_own = db->seed0;
  pr.key_prev = db->seed1;
  pr.nonce = nonce_of(db->code_length == (size_t)kIrisCodeLength ? kDomCodeDot : kDomMaskDot,
                      (uint32_t)db->dm->device);
  pr.batch = db->batch;
  pr.batch_dev = db->batch_from_device ? db->dm->d_batch : nullptr;
  return IRS_OK;
}

int irs_sharedb_dot_many(irs_sharedb* const* engines, const uint16_t* multipliers, int n, size_t offset, size_t len,
                         void* stream) {
  CHECK(engines && multipliers && n > 0 && n <= kMaxGemmProblems, IRS_ERR_INVALID, "1..6 engines per launch");
  irs_device_manager* dm = engines[0]->dm;
  CU(cudaSetDevice(dm->device));
  GemmParams P;
  memset(&P, 0, sizeof P);
  P.n_prob = n;
  P.err = dm->d_err;
  for (int i = 0; i < n; i++) {
    CHECK(engines[i] && engines[i]->dm == dm, IRS_ERR_INVALID, "engine %d missing or on another device", i);
    CHECK(engines[i]->block_n == engines[0]->block_n, IRS_ERR_INVALID, "engines need the same padded query length");
    CHECK(engines[i]->pair == engines[0]->pair, IRS_ERR_INVALID, "engines need the same GEMM variant (set_pair)");
    int rc = fill_problem(engines[i], multipliers[i], offset, len, P.prob[i]);
    if (rc) return rc;
  }
  cudaStream_t s = party_stream(dm, engines[0]->peer, stream);
  // The engines' inputs may have been written on their own party streams
  // (not while a graph is being captured: then all work is on the capture
  // stream and the uploads happened before the capture began).
  for (int i = 0; i < n; i++)
    if (!dm->capturing && dm->streams[engines[i]->peer] != s) {
      CU(cudaEventRecord(engines[i]->done, dm->streams[engines[i]->peer]));
      CU(cudaStreamWaitEvent(s, engines[i]->done, 0));
    }
  if (len) {
    if (dm->stall_limit_ns && !dm->capturing) {  // one-shot test hook
      P.test_stall = 1;
      P.wait_timeout_ns = dm->stall_limit_ns;
      dm->stall_limit_ns = 0;
    }
    StageTimer timer(dm, s, "dot");
    CU(launch_limb_gemm(P, engines[0]->block_n, engines[0]->pair, dm->n_sms, s));
  }
  for (int i = 0; i < n; i++) {
    engines[i]->res_offset = offset;
    engines[i]->res_len = len;
    if (!dm->capturing) CU(cudaEventRecord(engines[i]->done, s));  // a graph launch records graph_done instead
  }
  return IRS_OK;
}

int irs_sharedb_dot(irs_sharedb* db, size_t offset, size_t len, uint16_t multiplier, void* stream) {
  CHECK(db, IRS_ERR_INVALID, "db is NULL");
  irs_sharedb* e[1] = {db};
  uint16_t m[1] = {multiplier};
  return irs_sharedb_dot_many(e, m, 1, offset, len, stream ? stream : db->dm->streams[db->peer]);
}

int irs_sharedb_fetch_results(irs_sharedb* db, uint16_t* host, size_t len) {
  CHECK(db && host, IRS_ERR_INVALID, "bad arguments");
  CHECK(len <= db->res_len, IRS_ERR_STATE, "only %zu results available", db->res_len);
  irs_device_manager* dm = db->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[db->peer];
  std::vector<uint16_t> tmp(len * db->n_pad);
  CU(cudaMemcpyAsync(tmp.data(), db->results, tmp.size() * 2, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  int rc = check_device_error(dm);
  if (rc) return rc;
  for (size_t m = 0; m < len; m++)
    for (size_t q = 0; q < db->query_length; q++)
      host[q * len + m] = q < db->n_pad ? tmp[m * db->n_pad + q] : (uint16_t)0;
  return IRS_OK;
}

int irs_sharedb_result_view(irs_sharedb* db, const uint16_t** dev, size_t* row_stride) {
  CHECK(db && dev && row_stride, IRS_ERR_INVALID, "bad arguments");
  *dev = db->results;
  *row_stride = db->n_pad;
  return IRS_OK;
}

// ---------------------------------------------------------------------------
// Circuits
// ---------------------------------------------------------------------------
int irs_circuits_new(irs_device_manager* dm, const uint32_t seeds[3][2][8], irs_circuits** out) {
  CHECK(dm && seeds && out, IRS_ERR_INVALID, "bad arguments");
  *out = nullptr;
  for (int p = 0; p < 3; p++)
    CHECK(memcmp(seeds[p][1], seeds[(p + 2) % 3][0], 32) == 0, IRS_ERR_INVALID,
          "seed1 of party %d must equal seed0 of party %d", p, (p + 2) % 3);
  auto* c = new (std::nothrow) irs_circuits();
  CHECK(c, IRS_ERR_NOMEM, "host allocation failed");
  c->dm = dm;
  for (int p = 0; p < 3; p++) c->keys[p] = key_of(seeds[p][0]);
  *out = c;
  return IRS_OK;
}

int irs_circuits_destroy(irs_circuits* c) {
  delete c;
  return IRS_OK;
}

int irs_circuits_set_batch(irs_circuits* c, uint64_t batch_id) {
  CHECK(c, IRS_ERR_INVALID, "c is NULL");
  CHECK(batch_id < (1ull << 24), IRS_ERR_INVALID, "batch id must be below 2^24");
  c->batch = batch_id;
  return IRS_OK;
}

static void base_params(irs_circuits* c, ThresholdParams& P) {
  memset(&P, 0, sizeof P);
  for (int p = 0; p < 3; p++) P.key[p] = c->keys[p];
  P.nonce = nonce_of(kDomCircuit, (uint32_t)c->dm->device);
  P.batch = c->batch;
  P.batch_dev = c->batch_from_device ? c->dm->d_batch : nullptr;
}

// Splits [3][n/32] result components into each party's (a, b) u64 words.
__global__ void scatter_views_kernel(const uint32_t* comp, size_t n_words32, uint64_t* a0, uint64_t* a1, uint64_t* a2,
                                     uint64_t* b0, uint64_t* b1, uint64_t* b2, uint64_t* opened) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // u64 word
  if (2 * i >= n_words32) return;
  auto w64 = [&](int p) {
    const uint32_t* c = comp + (size_t)p * n_words32;
    return (uint64_t)c[2 * i] | ((uint64_t)c[2 * i + 1] << 32);
  };
  const uint64_t c0 = w64(0), c1 = w64(1), c2 = w64(2);
  if (a0) a0[i] = c0;
  if (a1) a1[i] = c1;
  if (a2) a2[i] = c2;
  if (b0) b0[i] = c2;
  if (b1) b1[i] = c0;
  if (b2) b2[i] = c1;
  if (opened) opened[i] = c0 ^ c1 ^ c2;
}

static int run_flat(irs_circuits* c, const uint16_t* const code_a[3], const uint16_t* const mask_a[3], size_t n,
                    uint32_t threshold_a, uint64_t* const res_a[3], uint64_t* const res_b[3], uint64_t* opened,
                    int stage, void* stream) {
  CHECK(c && code_a, IRS_ERR_INVALID, "bad arguments");
  CHECK(n % 64 == 0, IRS_ERR_INVALID, "n = %zu must be a multiple of 64", n);
  for (int p = 0; p < 3; p++) {
    CHECK(code_a[p] && (stage != kStageFull || (mask_a && mask_a[p])), IRS_ERR_INVALID, "share pointer missing");
    CHECK(((uintptr_t)code_a[p] & 15) == 0 && (stage != kStageFull || ((uintptr_t)mask_a[p] & 15) == 0),
          IRS_ERR_INVALID, "share pointers must be 16-byte aligned");
  }
  irs_device_manager* dm = c->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = party_stream(dm, 0, stream);
  ThresholdParams P;
  base_params(c, P);
  for (int p = 0; p < 3; p++) {
    P.code[p] = code_a[p];
    P.mask[p] = stage == kStageFull ? mask_a[p] : code_a[p];
  }
  P.threshold_a = threshold_a;
  P.n_words = n / 32;
  P.word_base = 0;
  uint32_t* comp = nullptr;
  void* p;
  int rc = pool_alloc(dm, 0, 3 * P.n_words * 4, &p);
  if (rc) return rc;
  comp = (uint32_t*)p;
  P.res_comp = comp;
  cudaError_t e = launch_threshold_flat(P, stage, s);
  if (e == cudaSuccess) {
    const size_t w64 = n / 64;
    scatter_views_kernel<<<(unsigned)((w64 + 255) / 256), 256, 0, s>>>(
        comp, P.n_words, res_a ? res_a[0] : nullptr, res_a ? res_a[1] : nullptr, res_a ? res_a[2] : nullptr,
        res_b ? res_b[0] : nullptr, res_b ? res_b[1] : nullptr, res_b ? res_b[2] : nullptr, opened);
    e = cudaGetLastError();
  }
  cudaFreeAsync(comp, s);
  if (e != cudaSuccess) return fail(IRS_ERR_CUDA, "threshold launch: %s", cudaGetErrorString(e));
  return IRS_OK;
}

int irs_circuits_compare_threshold_masked_many(irs_circuits* c, const uint16_t* const code_a[3],
                                               const uint16_t* const mask_a[3], size_t n, uint32_t threshold_a,
                                               uint64_t* const res_a[3], uint64_t* const res_b[3], uint64_t* opened,
                                               void* stream) {
  return run_flat(c, code_a, mask_a, n, threshold_a, res_a, res_b, opened, kStageFull, stream);
}

// The shared OR of the bit vector whose components are comp[p * n_words + w]
// (party p's a-share), into host out[4]: the three components and the opened
// bit.  Synchronous.
static int run_or_tree(irs_circuits* c, const uint32_t* comp, size_t n_words, uint32_t* out, cudaStream_t s) {
  irs_device_manager* dm = c->dm;
  OrTreeParams P;
  memset(&P, 0, sizeof P);
  for (int p = 0; p < 3; p++) P.key[p] = c->keys[p];
  P.nonce = nonce_of(kDomOrTree, (uint32_t)dm->device);
  P.batch = c->batch;
  P.batch_dev = c->batch_from_device ? dm->d_batch : nullptr;
  void* p;
  int rc = pool_alloc(dm, 0, (6 * n_words + 4) * 4, &p);
  if (rc) return rc;
  uint32_t* scratch = static_cast<uint32_t*>(p);
  uint32_t* out4 = scratch + 6 * n_words;
  cudaError_t e = launch_or_tree(P, comp, n_words, scratch, out4, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, out4, 16, cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(scratch, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(IRS_ERR_CUDA, "or tree: %s", cudaGetErrorString(e));
  return check_device_error(dm);
}

int irs_circuits_or_reduce(irs_circuits* c, const uint64_t* const res_a[3], size_t n, uint32_t out[4], void* stream) {
  CHECK(c && res_a && out, IRS_ERR_INVALID, "bad arguments");
  CHECK(n > 0 && n % 64 == 0, IRS_ERR_INVALID, "n = %zu must be a positive multiple of 64", n);
  for (int p = 0; p < 3; p++) CHECK(res_a[p], IRS_ERR_INVALID, "share pointer missing");
  irs_device_manager* dm = c->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = party_stream(dm, 0, stream);
  const size_t n_words = n / 32;
  // gather the three a-shares (u64 words = pairs of u32 words) into one [3][n_words] vector
  void* p;
  int rc = pool_alloc(dm, 0, 3 * n_words * 4, &p);
  if (rc) return rc;
  uint32_t* comp = static_cast<uint32_t*>(p);
  cudaError_t e = cudaSuccess;
  for (int q = 0; q < 3 && e == cudaSuccess; q++)
    e = cudaMemcpyAsync(comp + q * n_words, res_a[q], n_words * 4, cudaMemcpyDeviceToDevice, s);
  rc = e == cudaSuccess ? run_or_tree(c, comp, n_words, out, s) : fail(IRS_ERR_CUDA, "copy: %s", cudaGetErrorString(e));
  cudaFreeAsync(comp, s);
  return rc;
}

int irs_circuits_compare_threshold_masked_many_with_or_tree(irs_circuits* c, const uint16_t* const code_a[3],
                                                            const uint16_t* const mask_a[3], size_t n,
                                                            uint32_t threshold_a, uint32_t out[4], void* stream) {
  CHECK(c && code_a && mask_a && out, IRS_ERR_INVALID, "bad arguments");
  CHECK(n > 0 && n % 64 == 0, IRS_ERR_INVALID, "n = %zu must be a positive multiple of 64", n);
  for (int p = 0; p < 3; p++) {
    CHECK(code_a[p] && mask_a[p], IRS_ERR_INVALID, "share pointer missing");
    CHECK(((uintptr_t)code_a[p] & 15) == 0 && ((uintptr_t)mask_a[p] & 15) == 0, IRS_ERR_INVALID,
          "share pointers must be 16-byte aligned");
  }
  irs_device_manager* dm = c->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = party_stream(dm, 0, stream);
  ThresholdParams P;
  base_params(c, P);
  for (int p = 0; p < 3; p++) {
    P.code[p] = code_a[p];
    P.mask[p] = mask_a[p];
  }
  P.threshold_a = threshold_a;
  P.n_words = n / 32;
  void* p;
  int rc = pool_alloc(dm, 0, 3 * P.n_words * 4, &p);
  if (rc) return rc;
  P.res_comp = static_cast<uint32_t*>(p);
  cudaError_t e = launch_threshold_flat(P, kStageFull, s);
  rc = e == cudaSuccess ? run_or_tree(c, P.res_comp, P.n_words, out, s)
                        : fail(IRS_ERR_CUDA, "threshold launch: %s", cudaGetErrorString(e));
  cudaFreeAsync(P.res_comp, s);
  return rc;
}

int irs_circuits_extract_msb_of_code(irs_circuits* c, const uint16_t* const code_a[3], size_t n,
                                     uint64_t* const res_a[3], uint64_t* const res_b[3], uint64_t* opened,
                                     void* stream) {
  return run_flat(c, code_a, nullptr, n, 0, res_a, res_b, opened, kStageMsbOnly, stream);
}

int irs_circuits_lift_mpc(irs_circuits* c, const uint16_t* const mask_a[3], size_t n, uint16_t* const corr[3],
                          void* stream) {
  CHECK(c && mask_a && corr, IRS_ERR_INVALID, "bad arguments");
  CHECK(n % 64 == 0, IRS_ERR_INVALID, "n = %zu must be a multiple of 64", n);
  irs_device_manager* dm = c->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = party_stream(dm, 0, stream);
  ThresholdParams P;
  base_params(c, P);
  for (int p = 0; p < 3; p++) {
    CHECK(mask_a[p] && corr[p] && ((uintptr_t)mask_a[p] & 15) == 0, IRS_ERR_INVALID, "bad share pointer");
    P.mask[p] = mask_a[p];
    P.code[p] = mask_a[p];
  }
  P.n_words = n / 32;
  void* p;
  int rc = pool_alloc(dm, 0, 6 * n * 2, &p);
  if (rc) return rc;
  uint16_t* tmp = (uint16_t*)p;
  cudaError_t e = launch_lift_flat(P, tmp, s);
  for (int q = 0; q < 3 && e == cudaSuccess; q++)
    e = cudaMemcpyAsync(corr[q], tmp + (size_t)2 * q * n, 2 * n * 2, cudaMemcpyDeviceToDevice, s);
  cudaFreeAsync(tmp, s);
  if (e != cudaSuccess) return fail(IRS_ERR_CUDA, "lift launch: %s", cudaGetErrorString(e));
  return IRS_OK;
}

// ---------------------------------------------------------------------------
// DistanceComparator
// ---------------------------------------------------------------------------
constexpr uint32_t kMaxForced = 256;

// Buffer layout of the distance capture: [0] count, then entry [cap], row
// [cap], code [3][cap] u16, mask [3][cap] u16.
static void set_distance_capture(irs_distance_comparator* dc, ThresholdParams& P) {
  if (!dc->d_dist) return;
  const size_t cap = dc->dist_cap;
  P.dist_count = dc->d_dist;
  P.dist_entry = dc->d_dist + 1;
  P.dist_row = dc->d_dist + 1 + cap;
  P.dist_code = reinterpret_cast<uint16_t*>(dc->d_dist + 1 + 2 * cap);
  P.dist_mask = P.dist_code + 3 * cap;
  P.dist_cap = (uint32_t)cap;
  if (dc->d_forced && dc->n_forced) {
    P.forced_query = dc->d_forced;
    P.forced_entry = dc->d_forced + kMaxForced;
    P.n_forced = dc->n_forced;
  }
}

int irs_dc_init(irs_device_manager* dm, size_t max_queries, size_t max_db_length, size_t match_list_cap,
                irs_distance_comparator** out) {
  CHECK(dm && out && max_queries > 0 && max_db_length > 0, IRS_ERR_INVALID, "bad arguments");
  *out = nullptr;
  CU(cudaSetDevice(dm->device));
  auto* dc = new (std::nothrow) irs_distance_comparator();
  CHECK(dc, IRS_ERR_NOMEM, "host allocation failed");
  dc->dm = dm;
  dc->max_queries = max_queries;
  dc->max_db = max_db_length;
  dc->stride_bits = round_up(max_db_length, 64);
  dc->self_stride_bits = round_up(max_queries, 64);
  dc->match_cap = match_list_cap ? match_list_cap : 1;
  dc->slot_cap = 65536 / kSlotRows;
  dc->seg_cap = dc->slot_cap * 32;
  struct { void** p; size_t bytes; } allocs[] = {
      {(void**)&dc->bitmap, max_queries * dc->stride_bits / 8},
      {(void**)&dc->self_bitmap, max_queries * dc->self_stride_bits / 8},
      {(void**)&dc->match_list, dc->match_cap * 8},
      {(void**)&dc->counters, 16},
      {(void**)&dc->partial, max_db_length * 4},
      {(void**)&dc->final_results, max_queries * 4},
      {(void**)&dc->match_counters, max_queries * 4},
      {(void**)&dc->all_matches, max_queries * kMaxMatchesLen * 4},
      {(void**)&dc->d_slot_valid, dc->slot_cap * 4},
      {(void**)&dc->d_slot_query, dc->slot_cap * 4},
      {(void**)&dc->d_seg_start, (dc->slot_cap + 1) * 4},
      {(void**)&dc->d_seg_query, dc->slot_cap * 32 * 4},
      {(void**)&dc->d_seg_mask, dc->slot_cap * 32 * 4},
      {(void**)&dc->d_take, max_queries * (2 + kMaxMatchesLen) * 4},
  };
  for (auto& a : allocs) {
    cudaError_t e = cudaMalloc(a.p, a.bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      irs_dc_destroy(dc);
      return fail(IRS_ERR_NOMEM, "distance comparator allocation of %zu bytes failed", a.bytes);
    }
  }
  int rc = irs_dc_reset(dc, nullptr);
  if (rc) { irs_dc_destroy(dc); return rc; }
  CU(cudaStreamSynchronize(dm->streams[0]));
  *out = dc;
  return IRS_OK;
}

int irs_dc_destroy(irs_distance_comparator* dc) {
  if (!dc) return IRS_OK;
  cudaSetDevice(dc->dm->device);
  void* ps[] = {dc->bitmap, dc->self_bitmap, dc->match_list, dc->counters, dc->partial, dc->final_results,
                dc->match_counters, dc->all_matches, dc->d_slot_valid, dc->d_slot_query,
                dc->d_seg_start, dc->d_seg_query, dc->d_seg_mask, dc->d_take, dc->d_dist, dc->d_forced,
                dc->ring};
  for (void* p : ps) if (p) cudaFree(p);
  delete dc;
  return IRS_OK;
}

int irs_dc_reset(irs_distance_comparator* dc, void* stream) {
  CHECK(dc, IRS_ERR_INVALID, "dc is NULL");
  cudaStream_t s = party_stream(dc->dm, 0, stream);
  CU(cudaMemsetAsync(dc->bitmap, 0, dc->max_queries * dc->stride_bits / 8, s));
  CU(cudaMemsetAsync(dc->self_bitmap, 0, dc->max_queries * dc->self_stride_bits / 8, s));
  CU(cudaMemsetAsync(dc->counters, 0, 16, s));
  CU(cudaMemsetAsync(dc->final_results, 0xFF, dc->max_queries * 4, s));
  CU(cudaMemsetAsync(dc->match_counters, 0, dc->max_queries * 4, s));
  return IRS_OK;
}

int irs_dc_compare_threshold_open(irs_distance_comparator* dc, irs_circuits* c, irs_sharedb* const code_engines[3],
                                  irs_sharedb* const mask_engines[3], size_t offset, size_t len, size_t n_slots,
                                  const uint32_t* slot_valid, const uint32_t* slot_query, uint32_t threshold_a,
                                  int self_check, void* stream) {
  CHECK(dc && c && code_engines && mask_engines, IRS_ERR_INVALID, "bad arguments");
  CHECK(offset % 32 == 0, IRS_ERR_INVALID, "offset must be a multiple of 32");
  CHECK(n_slots <= dc->slot_cap, IRS_ERR_INVALID, "too many slots");
  const size_t n_pad = code_engines[0]->n_pad;
  CHECK(n_slots * kSlotRows <= n_pad, IRS_ERR_INVALID, "slots exceed the padded query rows");
  for (int p = 0; p < 3; p++) {
    CHECK(code_engines[p] && mask_engines[p], IRS_ERR_INVALID, "engine missing");
    CHECK(code_engines[p]->n_pad == n_pad && mask_engines[p]->n_pad == n_pad, IRS_ERR_INVALID,
          "engines need the same query padding");
    CHECK(code_engines[p]->res_offset == offset && mask_engines[p]->res_offset == offset &&
              code_engines[p]->res_len >= len && mask_engines[p]->res_len >= len,
          IRS_ERR_STATE, "engine results do not cover entries %zu..%zu", offset, offset + len);
  }
  const size_t stride_bits = self_check ? dc->self_stride_bits : dc->stride_bits;
  CHECK(offset + len <= stride_bits, IRS_ERR_INVALID, "entries exceed the bitmap width");
  irs_device_manager* dm = dc->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = party_stream(dm, 0, stream);
  // Receive: wait until every party's shares have been produced.
  // The GEMMs ran on another stream: wait for them (inside a graph capture
  // they are earlier nodes of the same capture stream).
  for (int p = 0; !dm->capturing && p < 3; p++) {
    CU(cudaStreamWaitEvent(s, code_engines[p]->done, 0));
    CU(cudaStreamWaitEvent(s, mask_engines[p]->done, 0));
  }
  ThresholdParams P;
  base_params(c, P);
  for (int p = 0; p < 3; p++) {
    P.code[p] = code_engines[p]->results;
    P.mask[p] = mask_engines[p]->results;
  }
  P.threshold_a = threshold_a;
  P.n_entries = (uint32_t)len;
  P.m0 = (uint32_t)offset;
  P.n_pad = (uint32_t)n_pad;
  P.n_slots = (uint32_t)n_slots;
  if (slot_valid) {
    CU(cudaMemcpyAsync(dc->d_slot_valid, slot_valid, n_slots * 4, cudaMemcpyHostToDevice, s));
    P.slot_valid = dc->d_slot_valid;
  }
  if (slot_query) {
    for (size_t i = 0; i < n_slots; i++)
      CHECK(slot_query[i] < dc->max_queries, IRS_ERR_INVALID, "slot %zu reports to query %u >= max", i, slot_query[i]);
    CU(cudaMemcpyAsync(dc->d_slot_query, slot_query, n_slots * 4, cudaMemcpyHostToDevice, s));
    P.slot_query = dc->d_slot_query;
  } else {
    CHECK(n_slots <= dc->max_queries, IRS_ERR_INVALID, "more slots than queries");
  }
  P.bitmap = self_check ? dc->self_bitmap : dc->bitmap;
  P.bitmap_stride = (uint32_t)stride_bits;
  P.match_count = dc->counters;
  P.match_list = self_check ? nullptr : dc->match_list;
  P.match_cap = (uint32_t)dc->match_cap;
  if (!self_check) set_distance_capture(dc, P);
  {
    StageTimer timer(dm, s, "threshold_open");
    CU(launch_threshold_bitmap(P, s));
  }
  if (slot_valid || slot_query) CU(cudaStreamSynchronize(s));  // host arrays are caller-owned
  return IRS_OK;
}

int irs_dc_set_segments(irs_distance_comparator* dc, size_t n_slots, const uint32_t* seg_start,
                        const uint32_t* seg_query, const uint32_t* seg_mask) {
  CHECK(dc && seg_start && n_slots > 0 && n_slots <= dc->slot_cap, IRS_ERR_INVALID, "bad arguments");
  CHECK(seg_start[0] == 0, IRS_ERR_INVALID, "seg_start[0] must be 0");
  for (size_t i = 0; i < n_slots; i++)
    CHECK(seg_start[i + 1] >= seg_start[i], IRS_ERR_INVALID, "seg_start must be non-decreasing");
  const size_t n_seg = seg_start[n_slots];
  CHECK(n_seg <= dc->seg_cap && (n_seg == 0 || (seg_query && seg_mask)), IRS_ERR_INVALID, "too many segments");
  for (size_t k = 0; k < n_seg; k++)
    CHECK(seg_query[k] < dc->max_queries, IRS_ERR_INVALID, "segment %zu reports to query %u >= max", k, seg_query[k]);
  irs_device_manager* dm = dc->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[0];
  CU(cudaMemcpyAsync(dc->d_seg_start, seg_start, (n_slots + 1) * 4, cudaMemcpyHostToDevice, s));
  if (n_seg) {
    CU(cudaMemcpyAsync(dc->d_seg_query, seg_query, n_seg * 4, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(dc->d_seg_mask, seg_mask, n_seg * 4, cudaMemcpyHostToDevice, s));
  }
  if (dm->host_sync) CU(cudaStreamSynchronize(s));  // the tables are caller-owned host memory
  dc->n_seg_slots = n_slots;
  dc->have_segments = true;
  return IRS_OK;
}

int irs_dc_compare_threshold_open_prepared(irs_distance_comparator* dc, irs_circuits* c,
                                           irs_sharedb* const code_engines[3], irs_sharedb* const mask_engines[3],
                                           size_t offset, size_t len, uint32_t threshold_a, int self_check,
                                           void* stream) {
  CHECK(dc && c && code_engines && mask_engines, IRS_ERR_INVALID, "bad arguments");
  CHECK(dc->have_segments, IRS_ERR_STATE, "irs_dc_set_segments not called");
  CHECK(offset % 32 == 0, IRS_ERR_INVALID, "offset must be a multiple of 32");
  const size_t n_pad = code_engines[0]->n_pad;
  CHECK(dc->n_seg_slots * kSlotRows <= n_pad, IRS_ERR_INVALID, "segment slots exceed the padded query rows");
  for (int p = 0; p < 3; p++) {
    CHECK(code_engines[p] && mask_engines[p], IRS_ERR_INVALID, "engine missing");
    CHECK(code_engines[p]->n_pad == n_pad && mask_engines[p]->n_pad == n_pad, IRS_ERR_INVALID,
          "engines need the same query padding");
    CHECK(code_engines[p]->res_offset == offset && mask_engines[p]->res_offset == offset &&
              code_engines[p]->res_len >= len && mask_engines[p]->res_len >= len,
          IRS_ERR_STATE, "engine results do not cover entries %zu..%zu", offset, offset + len);
  }
  const size_t stride_bits = self_check ? dc->self_stride_bits : dc->stride_bits;
  CHECK(offset + len <= stride_bits, IRS_ERR_INVALID, "entries exceed the bitmap width");
  irs_device_manager* dm = dc->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = party_stream(dm, 0, stream);
  // The GEMMs ran on another stream: wait for them (inside a graph capture
  // they are earlier nodes of the same capture stream).
  for (int p = 0; !dm->capturing && p < 3; p++) {
    CU(cudaStreamWaitEvent(s, code_engines[p]->done, 0));
    CU(cudaStreamWaitEvent(s, mask_engines[p]->done, 0));
  }
  ThresholdParams P;
  base_params(c, P);
  for (int p = 0; p < 3; p++) {
    P.code[p] = code_engines[p]->results;
    P.mask[p] = mask_engines[p]->results;
  }
  P.threshold_a = threshold_a;
  P.n_entries = (uint32_t)len;
  P.m0 = (uint32_t)offset;
  P.n_pad = (uint32_t)n_pad;
  P.n_slots = (uint32_t)dc->n_seg_slots;
  P.seg_start = dc->d_seg_start;
  P.seg_query = dc->d_seg_query;
  P.seg_mask = dc->d_seg_mask;
  P.bitmap = self_check ? dc->self_bitmap : dc->bitmap;
  P.bitmap_stride = (uint32_t)stride_bits;
  P.match_count = dc->counters;
  P.match_list = self_check ? nullptr : dc->match_list;
  P.match_cap = (uint32_t)dc->match_cap;
  if (!self_check) set_distance_capture(dc, P);
  {
    StageTimer timer(dm, s, "threshold_open");
    CU(launch_threshold_bitmap(P, s));
  }
  return IRS_OK;
}

int irs_dc_scan_fused(irs_distance_comparator* dc, irs_circuits* c, irs_sharedb* const code_engines[3],
                      irs_sharedb* const mask_engines[3], size_t offset, size_t len, size_t n_slots,
                      uint32_t threshold_a, int use_segments, void* stream) {
  CHECK(dc && c && code_engines && mask_engines, IRS_ERR_INVALID, "bad arguments");
  CHECK(offset % 32 == 0, IRS_ERR_INVALID, "offset must be a multiple of 32");
  irs_sharedb* eng[kFusedEngines] = {code_engines[0], code_engines[1], code_engines[2],
                                      mask_engines[0], mask_engines[1], mask_engines[2]};
  for (int e = 0; e < kFusedEngines; e++) {
    CHECK(eng[e] && eng[e]->dm == dc->dm, IRS_ERR_INVALID, "engine %d missing or on another device", e);
    CHECK(eng[e]->peer == e % 3, IRS_ERR_INVALID, "engine %d must belong to party %d", e, e % 3);
    CHECK(eng[e]->code_length == (size_t)(e < 3 ? kIrisCodeLength : kMaskCodeLength), IRS_ERR_INVALID,
          "engine %d has code length %zu", e, eng[e]->code_length);
  }
  const size_t n_pad = eng[0]->n_pad;
  for (int e = 1; e < kFusedEngines; e++)
    CHECK(eng[e]->n_pad == n_pad, IRS_ERR_INVALID, "engines need the same query padding");
  CHECK(n_pad % kFusedBlockN == 0, IRS_ERR_INVALID,
        "the fused scan needs padded query rows in multiples of %d (got %zu)", kFusedBlockN, n_pad);
  if (use_segments) {
    CHECK(dc->have_segments, IRS_ERR_STATE, "irs_dc_set_segments not called");
    n_slots = dc->n_seg_slots;
  } else {
    CHECK(n_slots <= dc->max_queries && n_slots <= dc->slot_cap, IRS_ERR_INVALID, "too many slots");
  }
  CHECK(n_slots * kSlotRows <= n_pad, IRS_ERR_INVALID, "slots exceed the padded query rows");
  CHECK(offset + len <= dc->stride_bits, IRS_ERR_INVALID, "entries exceed the bitmap width");
  irs_device_manager* dm = dc->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = party_stream(dm, 0, stream);
  FusedParams F;
  memset(&F, 0, sizeof F);
  const uint16_t mults[kFusedEngines] = {1, 1, 1, 2, 2, 2};
  for (int e = 0; e < kFusedEngines; e++) {
    int rc = fill_problem(eng[e], mults[e], offset, len, F.prob[e]);
    if (rc) return rc;
    // the fused kernel's query tile is 128 rows whatever the engine's own tile width
    if (make_tmap_u8(&F.prob[e].tm_b_lo, eng[e]->q_lo, eng[e]->n_cap, eng[e]->code_length, kFusedBlockN) ||
        make_tmap_u8(&F.prob[e].tm_b_hi, eng[e]->q_hi, eng[e]->n_cap, eng[e]->code_length, kFusedBlockN))
      return fail(IRS_ERR_CUDA, "tensor map for the query planes failed");
  }
  F.tiles_m = (int)((len + 127) / 128);
  F.tiles_n = (int)(n_pad / kFusedBlockN);
  F.total_work = F.tiles_m * F.tiles_n;
  F.err = dm->d_err;
  const size_t need = (size_t)dm->n_sms * kFusedRingBytesPerCta;  // the grid never exceeds one CTA per SM
  if (need > dc->ring_bytes) {
    // scratch for the dot shares of the CTAs' current tiles; allocated outside any capture
    CHECK(!dm->capturing, IRS_ERR_STATE,
          "the first fused scan of a comparator (which allocates its %zu-byte ring) must come before a graph capture",
          need);
    if (dc->ring) CU(cudaFree(dc->ring));
    dc->ring = nullptr;
    dc->ring_bytes = 0;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, need);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(IRS_ERR_NOMEM, "fused scan ring of %zu bytes: %s", need, cudaGetErrorString(e));
    }
    dc->ring = static_cast<uint16_t*>(p);
    dc->ring_bytes = need;
  }
  F.ring = dc->ring;
  ThresholdParams& T = F.T;
  base_params(c, T);
  T.threshold_a = threshold_a;
  T.n_entries = (uint32_t)len;
  T.m0 = (uint32_t)offset;
  T.n_pad = (uint32_t)n_pad;
  T.n_slots = (uint32_t)n_slots;
  if (use_segments) {
    T.seg_start = dc->d_seg_start;
    T.seg_query = dc->d_seg_query;
    T.seg_mask = dc->d_seg_mask;
  } else {
    CHECK(n_slots <= dc->max_queries, IRS_ERR_INVALID, "more slots than queries");
  }
  T.bitmap = dc->bitmap;
  T.bitmap_stride = (uint32_t)dc->stride_bits;
  T.match_count = dc->counters;
  T.match_list = dc->match_list;
  T.match_cap = (uint32_t)dc->match_cap;
  set_distance_capture(dc, T);
  // The engines' inputs may have been written on their own party streams.
  for (int e = 0; e < kFusedEngines; e++)
    if (!dm->capturing && dm->streams[eng[e]->peer] != s) {
      CU(cudaEventRecord(eng[e]->done, dm->streams[eng[e]->peer]));
      CU(cudaStreamWaitEvent(s, eng[e]->done, 0));
    }
  if (len && n_slots) {
    StageTimer timer(dm, s, "scan_fused");
    CU(launch_fused_scan(F, dm->n_sms, s));
  }
  for (int e = 0; e < kFusedEngines; e++) {
    eng[e]->res_offset = offset;
    eng[e]->res_len = 0;  // the dot shares stayed in the ring: no buffered results
    if (!dm->capturing) CU(cudaEventRecord(eng[e]->done, s));
  }
  return IRS_OK;
}

// ---------------------------------------------------------------------------
// CUDA graphs
// ---------------------------------------------------------------------------
int irs_graph_begin_capture(irs_device_manager* dm) {
  CHECK(dm, IRS_ERR_INVALID, "dm is NULL");
  CHECK(!dm->capturing, IRS_ERR_STATE, "a capture is already open");
  CU(cudaSetDevice(dm->device));
  CU(cudaStreamBeginCapture(dm->streams[0], cudaStreamCaptureModeThreadLocal));
  dm->capturing = true;
  return IRS_OK;
}

int irs_graph_end_capture(irs_device_manager* dm, irs_graph** out) {
  CHECK(dm && out, IRS_ERR_INVALID, "bad arguments");
  CHECK(dm->capturing, IRS_ERR_STATE, "no capture is open");
  *out = nullptr;
  dm->capturing = false;
  cudaGraph_t g = nullptr;
  CU(cudaStreamEndCapture(dm->streams[0], &g));
  auto* gr = new (std::nothrow) irs_graph();
  if (!gr) {
    cudaGraphDestroy(g);
    return fail(IRS_ERR_NOMEM, "host allocation failed");
  }
  gr->graph = g;
  gr->dm = dm;
  cudaError_t e = cudaGraphInstantiate(&gr->exec, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    delete gr;
    return fail(IRS_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
  }
  *out = gr;
  return IRS_OK;
}

int irs_graph_launch(irs_graph* g, void* stream) {
  CHECK(g && g->exec, IRS_ERR_INVALID, "graph is NULL");
  CU(cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)));
  // later query uploads on other party streams wait for the graph's GEMMs
  CU(cudaEventRecord(g->dm->graph_done, static_cast<cudaStream_t>(stream)));
  return IRS_OK;
}

int irs_graph_destroy(irs_graph* g) {
  if (!g) return IRS_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return IRS_OK;
}

int irs_dc_take_rows(irs_distance_comparator* dc, const uint32_t* rows, size_t n, size_t db_len, int clear,
                     uint32_t* counts, uint32_t* ids) {
  CHECK(dc && (n == 0 || (rows && counts && ids)), IRS_ERR_INVALID, "bad arguments");
  CHECK(n <= dc->max_queries, IRS_ERR_INVALID, "%zu rows exceed the comparator's %zu", n, dc->max_queries);
  CHECK(db_len <= dc->stride_bits, IRS_ERR_INVALID, "db_len %zu exceeds the bitmap width", db_len);
  for (size_t i = 0; i < n; i++)
    CHECK(rows[i] < dc->max_queries, IRS_ERR_INVALID, "row %u out of range", rows[i]);
  if (!n) return IRS_OK;
  irs_device_manager* dm = dc->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[0];
  uint32_t* d_rows = dc->d_take;
  uint32_t* d_counts = d_rows + dc->max_queries;
  uint32_t* d_ids = d_counts + dc->max_queries;
  CU(cudaMemcpyAsync(d_rows, rows, n * 4, cudaMemcpyHostToDevice, s));
  CU(launch_take_rows(dc->bitmap, (uint32_t)(dc->stride_bits / 32), d_rows, (uint32_t)n, (uint32_t)db_len, clear,
                      d_counts, d_ids, kMaxMatchesLen, s));
  CU(cudaMemcpyAsync(counts, d_counts, n * 4, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(ids, d_ids, n * kMaxMatchesLen * 4, cudaMemcpyDeviceToHost, s));
  if (!dm->host_sync) return IRS_OK;  // outputs valid once the stream passes the copies
  CU(cudaStreamSynchronize(s));
  return check_device_error(dm);
}

static size_t dist_bytes(size_t cap) { return (1 + 2 * cap) * 4 + 6 * cap * 2 + 16; }

int irs_dc_enable_distance_capture(irs_distance_comparator* dc, size_t cap) {
  CHECK(dc && cap > 0 && cap < (1u << 30), IRS_ERR_INVALID, "bad arguments");
  irs_device_manager* dm = dc->dm;
  CU(cudaSetDevice(dm->device));
  CU(cudaStreamSynchronize(dm->streams[0]));
  if (dc->d_dist) {
    cudaFree(dc->d_dist);
    dc->d_dist = nullptr;
  }
  void* p = nullptr;
  if (cudaMalloc(&p, dist_bytes(cap)) != cudaSuccess) {
    cudaGetLastError();
    return fail(IRS_ERR_NOMEM, "distance capture allocation of %zu bytes failed", dist_bytes(cap));
  }
  dc->d_dist = static_cast<uint32_t*>(p);
  dc->dist_cap = cap;
  CU(cudaMemset(dc->d_dist, 0, 4));
  return IRS_OK;
}

int irs_dc_set_forced_distances(irs_distance_comparator* dc, const uint32_t* query, const uint32_t* entry, size_t n) {
  CHECK(dc && (n == 0 || (query && entry)), IRS_ERR_INVALID, "bad arguments");
  CHECK(dc->d_dist, IRS_ERR_STATE, "distance capture not enabled");
  CHECK(n <= kMaxForced, IRS_ERR_INVALID, "%zu forced pairs exceed %u", n, kMaxForced);
  for (size_t i = 0; i < n; i++)
    CHECK(query[i] < dc->max_queries && entry[i] < dc->max_db, IRS_ERR_INVALID, "forced pair %zu out of range", i);
  irs_device_manager* dm = dc->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[0];
  if (!dc->d_forced) {
    void* p = nullptr;
    if (cudaMalloc(&p, 2 * kMaxForced * 4) != cudaSuccess) {
      cudaGetLastError();
      return fail(IRS_ERR_NOMEM, "forced-pair table allocation failed");
    }
    dc->d_forced = static_cast<uint32_t*>(p);
  }
  if (n) {
    CU(cudaMemcpyAsync(dc->d_forced, query, n * 4, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(dc->d_forced + kMaxForced, entry, n * 4, cudaMemcpyHostToDevice, s));
    CU(cudaStreamSynchronize(s));  // caller-owned host memory
  }
  dc->n_forced = (uint32_t)n;
  return IRS_OK;
}

int irs_dc_fetch_distances(irs_distance_comparator* dc, size_t cap, uint32_t* entry, uint32_t* row, uint16_t* code,
                           uint16_t* mask, size_t* n, int reset) {
  CHECK(dc && n, IRS_ERR_INVALID, "bad arguments");
  CHECK(dc->d_dist, IRS_ERR_STATE, "distance capture not enabled");
  irs_device_manager* dm = dc->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[0];
  uint32_t count = 0;
  CU(cudaMemcpyAsync(&count, dc->d_dist, 4, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  *n = count;  // may exceed the capture capacity: records beyond it were dropped
  const size_t k = std::min<size_t>(std::min<size_t>(count, dc->dist_cap), cap);
  const size_t dcap = dc->dist_cap;
  if (k) {
    CHECK(entry && row && code && mask, IRS_ERR_INVALID, "output arrays missing");
    CU(cudaMemcpyAsync(entry, dc->d_dist + 1, k * 4, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(row, dc->d_dist + 1 + dcap, k * 4, cudaMemcpyDeviceToHost, s));
    const uint16_t* dcode = reinterpret_cast<const uint16_t*>(dc->d_dist + 1 + 2 * dcap);
    for (int p = 0; p < 3; p++) {
      CU(cudaMemcpyAsync(code + p * cap, dcode + p * dcap, k * 2, cudaMemcpyDeviceToHost, s));
      CU(cudaMemcpyAsync(mask + p * cap, dcode + (3 + p) * dcap, k * 2, cudaMemcpyDeviceToHost, s));
    }
  }
  if (reset) CU(cudaMemsetAsync(dc->d_dist, 0, 4, s));
  CU(cudaStreamSynchronize(s));
  return check_device_error(dm);
}

int irs_dc_clear_rows(irs_distance_comparator* dc, size_t first, size_t n, void* stream) {
  CHECK(dc && first + n <= dc->max_queries, IRS_ERR_INVALID, "rows out of range");
  cudaStream_t s = party_stream(dc->dm, 0, stream);
  const size_t words = dc->stride_bits / 32;
  CU(cudaMemsetAsync(dc->bitmap + first * words, 0, n * words * 4, s));
  return IRS_OK;
}

int irs_dc_fetch_rows(irs_distance_comparator* dc, size_t first, size_t n, uint32_t* host, size_t cap_words,
                      size_t* row_words) {
  CHECK(dc && host && row_words && first + n <= dc->max_queries, IRS_ERR_INVALID, "bad arguments");
  const size_t words = dc->stride_bits / 32;
  *row_words = words;
  CHECK(n * words <= cap_words, IRS_ERR_INVALID, "host buffer holds %zu words, %zu needed", cap_words, n * words);
  irs_device_manager* dm = dc->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[0];
  if (n) {
    CU(cudaMemcpyAsync(host, dc->bitmap + first * words, n * words * 4, cudaMemcpyDeviceToHost, s));
    if (!dm->host_sync) return IRS_OK;  // rows valid once the stream passes the copy
    CU(cudaStreamSynchronize(s));
  }
  return check_device_error(dm);
}

int irs_dc_fetch_bitmap(irs_distance_comparator* dc, size_t n_queries, size_t db_len, uint64_t* host) {
  CHECK(dc && host && n_queries <= dc->max_queries && db_len <= dc->stride_bits, IRS_ERR_INVALID, "bad arguments");
  irs_device_manager* dm = dc->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[0];
  std::vector<uint32_t> tmp(n_queries * dc->stride_bits / 32);
  CU(cudaMemcpyAsync(tmp.data(), dc->bitmap, tmp.size() * 4, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  int rc = check_device_error(dm);
  if (rc) return rc;
  const size_t words = (n_queries * db_len + 63) / 64;
  memset(host, 0, words * 8);
  for (size_t q = 0; q < n_queries; q++)
    for (size_t e = 0; e < db_len; e++) {
      const uint32_t bit = (tmp[q * (dc->stride_bits / 32) + e / 32] >> (e % 32)) & 1u;
      if (bit) {
        const size_t o = q * db_len + e;
        host[o / 64] |= 1ull << (o % 64);
      }
    }
  return IRS_OK;
}

int irs_dc_fetch_matches(irs_distance_comparator* dc, uint32_t* pairs, size_t cap, size_t* n) {
  CHECK(dc && n && (pairs || !cap), IRS_ERR_INVALID, "bad arguments");
  irs_device_manager* dm = dc->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[0];
  uint32_t count = 0;
  CU(cudaMemcpyAsync(&count, dc->counters, 4, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  *n = count;
  const size_t avail = std::min<size_t>(std::min<size_t>(count, dc->match_cap), cap);
  if (avail) {
    CU(cudaMemcpyAsync(pairs, dc->match_list, avail * 8, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
  }
  int rc = check_device_error(dm);
  if (rc) return rc;
  if (count > dc->match_cap) return fail(IRS_ERR_OVERFLOW, "%u matches exceed the list capacity %zu", count, dc->match_cap);
  return IRS_OK;
}

int irs_dc_get_partial_results(irs_distance_comparator* dc, size_t n_queries, size_t db_len, uint32_t* ids, size_t cap,
                               size_t* n) {
  CHECK(dc && n && (ids || !cap) && n_queries <= dc->max_queries && db_len <= dc->max_db, IRS_ERR_INVALID,
        "bad arguments");
  irs_device_manager* dm = dc->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[0];
  CU(cudaMemsetAsync(dc->counters + 1, 0, 4, s));
  CU(launch_compact(dc->bitmap, (uint32_t)n_queries, (uint32_t)db_len, (uint32_t)(dc->stride_bits / 32), dc->partial,
                    dc->counters + 1, (uint32_t)dc->max_db, s));
  uint32_t count = 0;
  CU(cudaMemcpyAsync(&count, dc->counters + 1, 4, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  std::vector<uint32_t> tmp(std::min<size_t>(count, dc->max_db));
  if (!tmp.empty()) {
    CU(cudaMemcpyAsync(tmp.data(), dc->partial, tmp.size() * 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
  }
  std::sort(tmp.begin(), tmp.end());
  tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
  *n = tmp.size();
  const size_t k = std::min(cap, tmp.size());
  if (k) memcpy(ids, tmp.data(), k * 4);
  if (tmp.size() > cap) return fail(IRS_ERR_OVERFLOW, "%zu ids exceed cap %zu", tmp.size(), cap);
  return IRS_OK;
}

int irs_dc_join_db_matches(irs_distance_comparator* dc, irs_distance_comparator* right, const uint32_t* or_policy,
                           size_t n_queries, size_t db_len, void* stream) {
  CHECK(dc && n_queries <= dc->max_queries && db_len <= dc->max_db, IRS_ERR_INVALID, "bad arguments");
  CHECK(!right || right->stride_bits == dc->stride_bits, IRS_ERR_INVALID, "comparators differ in bitmap width");
  cudaStream_t s = party_stream(dc->dm, 0, stream);
  CU(launch_merge_db(dc->bitmap, right ? right->bitmap : nullptr, or_policy, (uint32_t)n_queries, (uint32_t)db_len,
                     (uint32_t)(dc->stride_bits / 32), dc->final_results, dc->match_counters, dc->all_matches, s));
  return IRS_OK;
}

int irs_dc_join_batch_matches(irs_distance_comparator* dc, irs_distance_comparator* right, size_t n_queries,
                              void* stream) {
  CHECK(dc && n_queries <= dc->max_queries, IRS_ERR_INVALID, "bad arguments");
  CHECK(!right || right->self_stride_bits == dc->self_stride_bits, IRS_ERR_INVALID, "comparators differ");
  cudaStream_t s = party_stream(dc->dm, 0, stream);
  CU(launch_merge_batch(dc->self_bitmap, right ? right->self_bitmap : nullptr, (uint32_t)n_queries,
                        (uint32_t)(dc->self_stride_bits / 32), dc->final_results, dc->match_counters,
                        dc->all_matches, s));
  return IRS_OK;
}

int irs_dc_fetch_final_results(irs_distance_comparator* dc, size_t n_queries, uint32_t* final_results,
                               uint32_t* match_counters, uint32_t* all_matches) {
  CHECK(dc && n_queries <= dc->max_queries, IRS_ERR_INVALID, "bad arguments");
  irs_device_manager* dm = dc->dm;
  CU(cudaSetDevice(dm->device));
  cudaStream_t s = dm->streams[0];
  if (final_results) CU(cudaMemcpyAsync(final_results, dc->final_results, n_queries * 4, cudaMemcpyDeviceToHost, s));
  if (match_counters) CU(cudaMemcpyAsync(match_counters, dc->match_counters, n_queries * 4, cudaMemcpyDeviceToHost, s));
  if (all_matches)
    CU(cudaMemcpyAsync(all_matches, dc->all_matches, n_queries * kMaxMatchesLen * 4, cudaMemcpyDeviceToHost, s));
  if (!dm->host_sync) return IRS_OK;  // outputs valid once the stream passes the copies
  CU(cudaStreamSynchronize(s));
  return check_device_error(dm);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Internal accessors (internal.h)
// ---------------------------------------------------------------------------
namespace irs {

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

int circuit_view(irs_circuits* c, CircuitView* v) {
  if (!c || !v) return set_error(IRS_ERR_INVALID, "circuits handle is NULL");
  for (int p = 0; p < 3; p++) v->keys[p] = c->keys[p];
  v->nonce = nonce_of(kDomCircuit, (uint32_t)c->dm->device);
  v->batch = c->batch;
  v->batch_dev = c->batch_from_device ? c->dm->d_batch : nullptr;
  v->device = c->dm->device;
  v->stream0 = c->dm->streams[0];
  return IRS_OK;
}

}  // namespace irs
