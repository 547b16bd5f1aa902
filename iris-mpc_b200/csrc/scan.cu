// The plain drop-in's DB pass and its autotuner (irs_scan_*).
//
// The reference's actor scans the share DB in chunks (DB_CHUNK_SIZE per
// device, iris-mpc-gpu/src/server/actor.rs:2246-2589): per chunk the dot
// products of the three parties' code and mask shares (Phase 1), then the
// threshold protocol, the open and the rotation OR (Phase 2).  An irs_scan
// runs that pass over the library's resident engines for one uploaded batch of
// 32-row query slots, along one of three paths per chunk: the one-SM limb GEMM
// launch then the threshold launch (IRS_SCAN_SPLIT), the same with the two-SM
// GEMM (IRS_SCAN_PAIR), or the one-kernel fused scan (IRS_SCAN_FUSED).
// irs_scan_tune picks the path, the GEMM tile width and the chunk length by
// timing every candidate on the batch at hand -- the choice cuBLAS makes
// internally for the reference's dot products, here made on the whole pass
// because under the B200's power cap the best GEMM depends on what runs beside
// it.  Results are identical on every path.
#include <algorithm>
#include <chrono>
#include <vector>
#include "internal.h"

struct irs_scan {
  irs_device_manager* dm = nullptr;
  irs_distance_comparator* dc = nullptr;
  irs_circuits* c = nullptr;
  irs_sharedb* ce[3] = {nullptr, nullptr, nullptr};
  irs_sharedb* me[3] = {nullptr, nullptr, nullptr};
  irs_sharedb* all[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  size_t n_slots = 0, db_len = 0;
  size_t n_rows = 0;      // padded query rows the candidates are for (0: n_slots x 32)
  bool segments = false;  // threshold via the comparator's stored segment table
  uint32_t threshold_a = 0;
  irs_scan_candidate cand{IRS_SCAN_SPLIT, 0, 65536};
  // per-chunk timing events (irs_scan_set_timing): per pass, the start and
  // then, per chunk, the end of its GEMM and the end of its threshold launch
  std::vector<cudaEvent_t> ev;
  size_t max_passes = 0, per_pass = 0, passes = 0;
};

namespace {

using irs::set_error;

constexpr uint64_t kChunks[] = {131072, 65536, 32768, 16384, 8192};
const uint16_t kMults[6] = {1, 1, 1, 2, 2, 2};

size_t n_chunks(const irs_scan* s) {
  return s->db_len ? (s->db_len + s->cand.chunk - 1) / s->cand.chunk : 0;
}

void free_events(irs_scan* s) {
  for (cudaEvent_t e : s->ev)
    if (e) cudaEventDestroy(e);
  s->ev.clear();
  s->max_passes = s->per_pass = s->passes = 0;
}

int timed_passes(irs_scan* s, const irs_scan_candidate& cand, int passes, double* ms) {
  int rc = irs_scan_configure(s, cand.path, cand.tile, cand.chunk);
  if (rc) return rc;
  // a warm pass, then `passes` consecutive ones: the power-capped clock
  // settles differently for long launches and for alternating GEMM /
  // threshold chunks, and a single pass after idle time does not show it
  if ((rc = irs_dc_reset(s->dc, nullptr)) || (rc = irs_scan_run(s, nullptr)) ||
      (rc = irs_device_manager_synchronize(s->dm)))
    return rc;
  const auto t0 = std::chrono::steady_clock::now();
  for (int i = 0; i < passes; i++)
    if ((rc = irs_dc_reset(s->dc, nullptr)) || (rc = irs_scan_run(s, nullptr))) return rc;
  if ((rc = irs_device_manager_synchronize(s->dm))) return rc;
  *ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / passes;
  return IRS_OK;
}

}  // namespace

extern "C" {

int irs_scan_init(irs_device_manager* dm, irs_distance_comparator* dc, irs_circuits* c,
                  irs_sharedb* const code_engines[3], irs_sharedb* const mask_engines[3], size_t n_slots,
                  size_t db_len, uint32_t threshold_a, irs_scan** out) {
  if (!out) return set_error(IRS_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (!dm || !dc || !c || !code_engines || !mask_engines) return set_error(IRS_ERR_INVALID, "bad arguments");
  if (!n_slots) return set_error(IRS_ERR_INVALID, "n_slots must be positive");
  irs_scan* s = new irs_scan;
  s->dm = dm;
  s->dc = dc;
  s->c = c;
  for (int p = 0; p < 3; p++) {
    if (!code_engines[p] || !mask_engines[p]) {
      delete s;
      return set_error(IRS_ERR_INVALID, "engine of party %d missing", p);
    }
    s->ce[p] = s->all[p] = code_engines[p];
    s->me[p] = s->all[3 + p] = mask_engines[p];
  }
  s->n_slots = n_slots;
  s->db_len = db_len;
  s->threshold_a = threshold_a;
  *out = s;
  return IRS_OK;
}

int irs_scan_destroy(irs_scan* s) {
  if (!s) return IRS_OK;
  free_events(s);
  delete s;
  return IRS_OK;
}

int irs_scan_candidates(irs_scan* s, irs_scan_candidate* out, size_t cap, size_t* n) {
  if (!s || !n || (cap && !out)) return set_error(IRS_ERR_INVALID, "bad arguments");
  const uint64_t rows = s->n_rows ? (uint64_t)s->n_rows : (uint64_t)s->n_slots * IRS_SLOT_ROWS;
  const uint64_t n_pad = (rows + 63) / 64 * 64;
  const uint64_t full = (s->db_len + 31) / 32 * 32;
  std::vector<uint64_t> chunks;
  for (uint64_t c : kChunks) {
    const uint64_t ch = std::max<uint64_t>(32, std::min(full, c));
    if (std::find(chunks.begin(), chunks.end(), ch) == chunks.end()) chunks.push_back(ch);
  }
  std::vector<int> tiles;
  for (int t : {256, 128, 64})
    if (n_pad % t == 0 && (t != 64 || n_pad <= 768)) tiles.push_back(t);
  if (tiles.empty()) tiles.push_back(64);
  std::vector<irs_scan_candidate> v;
  for (int t : tiles)
    for (uint64_t ch : chunks) v.push_back({IRS_SCAN_SPLIT, t, ch});
  if (n_pad % 256 == 0)
    for (uint64_t ch : chunks) v.push_back({IRS_SCAN_PAIR, 256, ch});
  if (n_pad % 128 == 0)  // the fused kernel on the three longest chunks
    for (size_t i = 0; i < chunks.size() && i < 3; i++) v.push_back({IRS_SCAN_FUSED, 128, chunks[i]});
  *n = v.size();
  for (size_t i = 0; i < v.size() && i < cap; i++) out[i] = v[i];
  return IRS_OK;
}

int irs_scan_configure(irs_scan* s, int path, int tile, size_t chunk) {
  if (!s) return set_error(IRS_ERR_INVALID, "scan is NULL");
  if (path != IRS_SCAN_SPLIT && path != IRS_SCAN_PAIR && path != IRS_SCAN_FUSED)
    return set_error(IRS_ERR_INVALID, "path %d is not IRS_SCAN_SPLIT, _PAIR or _FUSED", path);
  if (!chunk || chunk % 32) return set_error(IRS_ERR_INVALID, "chunk %zu must be a positive multiple of 32", chunk);
  if (path == IRS_SCAN_PAIR && tile != 256) return set_error(IRS_ERR_INVALID, "the two-SM GEMM runs the 256-row tile");
  for (irs_sharedb* e : s->all) {
    int rc = irs_sharedb_set_pair(e, path == IRS_SCAN_PAIR);
    if (!rc) rc = irs_sharedb_set_tile(e, path == IRS_SCAN_FUSED ? 0 : tile);
    if (rc) return rc;
  }
  if (path == IRS_SCAN_FUSED) {  // allocates the comparator's ring before any capture
    int rc = irs_dc_scan_fused(s->dc, s->c, s->ce, s->me, 0, 0, s->n_slots, s->threshold_a, s->segments, nullptr);
    if (rc) return rc;
  }
  s->cand = {path, tile, (uint64_t)chunk};
  free_events(s);  // the timing events are laid out for a chunk count
  return IRS_OK;
}

int irs_scan_set_rows(irs_scan* s, size_t n_rows, int use_segments) {
  if (!s) return set_error(IRS_ERR_INVALID, "scan is NULL");
  s->n_rows = n_rows;
  s->segments = use_segments != 0;
  return IRS_OK;
}

int irs_scan_current(irs_scan* s, irs_scan_candidate* cand) {
  if (!s || !cand) return set_error(IRS_ERR_INVALID, "bad arguments");
  *cand = s->cand;
  return IRS_OK;
}

int irs_scan_run(irs_scan* s, void* stream) {
  if (!s) return set_error(IRS_ERR_INVALID, "scan is NULL");
  void* st = stream;
  if (!st) {
    int rc = irs_device_manager_stream(s->dm, 0, &st);
    if (rc) return rc;
  }
  cudaStream_t cs = static_cast<cudaStream_t>(st);
  const size_t nc = n_chunks(s);
  // a timed pass counts once all its launches are enqueued; a failed one
  // leaves its slot to the next pass
  cudaEvent_t* ev = nullptr;
  if (s->per_pass && s->passes < s->max_passes) {
    ev = &s->ev[s->passes * s->per_pass];
    if (cudaEventRecord(ev[0], cs) != cudaSuccess) {
      cudaGetLastError();
      return set_error(IRS_ERR_CUDA, "timing event record failed");
    }
  }
  for (size_t k = 0; k < nc; k++) {
    const size_t off = k * s->cand.chunk;
    const size_t len = std::min<size_t>(s->cand.chunk, s->db_len - off);
    int rc;
    if (s->cand.path == IRS_SCAN_FUSED) {
      rc = irs_dc_scan_fused(s->dc, s->c, s->ce, s->me, off, len, s->n_slots, s->threshold_a, s->segments, st);
      if (!rc && ev) cudaEventRecord(ev[1 + 2 * k], cs);
    } else {
      rc = irs_sharedb_dot_many(s->all, kMults, 6, off, len, st);
      if (!rc && ev) cudaEventRecord(ev[1 + 2 * k], cs);
      if (!rc)
        rc = s->segments ? irs_dc_compare_threshold_open_prepared(s->dc, s->c, s->ce, s->me, off, len,
                                                                  s->threshold_a, 0, st)
                         : irs_dc_compare_threshold_open(s->dc, s->c, s->ce, s->me, off, len, s->n_slots, nullptr,
                                                         nullptr, s->threshold_a, 0, st);
    }
    if (rc) return rc;
    if (ev) cudaEventRecord(ev[2 + 2 * k], cs);
  }
  if (ev) s->passes++;
  return IRS_OK;
}

int irs_scan_set_timing(irs_scan* s, size_t max_passes) {
  if (!s) return set_error(IRS_ERR_INVALID, "scan is NULL");
  free_events(s);
  if (!max_passes) return IRS_OK;
  const size_t per = 1 + 2 * n_chunks(s);
  s->ev.assign(max_passes * per, nullptr);
  for (cudaEvent_t& e : s->ev)
    if (cudaEventCreate(&e) != cudaSuccess) {
      cudaGetLastError();
      e = nullptr;
      free_events(s);
      return set_error(IRS_ERR_CUDA, "creating %zu timing events failed", max_passes * per);
    }
  s->max_passes = max_passes;
  s->per_pass = per;
  return IRS_OK;
}

int irs_scan_timings(irs_scan* s, double* gemm_ms, double* threshold_ms, double* pass_ms, size_t cap, size_t* n,
                     int reset) {
  if (!s || !n || (cap && (!gemm_ms || !threshold_ms || !pass_ms))) return set_error(IRS_ERR_INVALID, "bad arguments");
  *n = s->passes;
  const size_t nc = s->per_pass ? (s->per_pass - 1) / 2 : 0;
  for (size_t p = 0; p < s->passes && p < cap; p++) {
    cudaEvent_t* ev = &s->ev[p * s->per_pass];
    if (cudaEventSynchronize(ev[2 * nc]) != cudaSuccess) {
      cudaGetLastError();
      return set_error(IRS_ERR_CUDA, "timing event wait failed");
    }
    double g = 0.0, t = 0.0;
    float x = 0.0f, y = 0.0f;
    bool ok = true;
    for (size_t k = 0; k < nc; k++) {
      ok = ok && cudaEventElapsedTime(&x, ev[2 * k], ev[1 + 2 * k]) == cudaSuccess;  // GEMM (or the fused launch)
      ok = ok && cudaEventElapsedTime(&y, ev[1 + 2 * k], ev[2 + 2 * k]) == cudaSuccess;  // threshold, open, OR
      g += x;
      t += y;
    }
    ok = ok && cudaEventElapsedTime(&x, ev[0], ev[2 * nc]) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      return set_error(IRS_ERR_CUDA, "reading the timing events of pass %zu failed", p);
    }
    gemm_ms[p] = g;
    threshold_ms[p] = t;
    pass_ms[p] = x;
  }
  if (reset) s->passes = 0;
  return IRS_OK;
}

int irs_scan_tune(irs_scan* s, int passes, int finalists, int rounds, int only_path, irs_scan_candidate* chosen,
                  irs_scan_timing* log, size_t log_cap, size_t* n_log) {
  if (!s || !chosen || (log_cap && !log)) return set_error(IRS_ERR_INVALID, "bad arguments");
  if (passes < 1 || finalists < 1 || rounds < 0) return set_error(IRS_ERR_INVALID, "passes, finalists >= 1, rounds >= 0");
  size_t nc = 0;
  int rc = irs_scan_candidates(s, nullptr, 0, &nc);
  if (rc) return rc;
  std::vector<irs_scan_candidate> cands(nc);
  if ((rc = irs_scan_candidates(s, cands.data(), nc, &nc))) return rc;
  if (only_path >= 0) {
    std::vector<irs_scan_candidate> keep;
    for (const irs_scan_candidate& c : cands)
      if (c.path == only_path) keep.push_back(c);
    if (keep.empty()) return set_error(IRS_ERR_INVALID, "no candidate on path %d for this batch shape", only_path);
    cands.swap(keep);
    nc = cands.size();
  }
  size_t nl = 0;
  auto note = [&](const irs_scan_candidate& c, double ms, int finalist) {
    if (nl < log_cap) log[nl] = {c, ms, finalist, 0};
    nl++;
  };
  // every candidate once
  std::vector<std::pair<double, size_t>> first;
  for (size_t i = 0; i < nc; i++) {
    double ms = 0.0;
    if ((rc = timed_passes(s, cands[i], passes, &ms))) return rc;
    first.push_back({ms, i});
    note(cands[i], ms, 0);
  }
  std::stable_sort(first.begin(), first.end(),
                   [](const std::pair<double, size_t>& a, const std::pair<double, size_t>& b) { return a.first < b.first; });
  const size_t nt = std::min<size_t>((size_t)finalists, first.size());
  irs_scan_candidate best = cands[first[0].second];
  // the fastest again, interleaved: the clock drifts over a tuning run by as
  // much as the candidates differ, so candidates timed far apart do not compare
  if (nt > 1 && rounds > 0) {
    std::vector<double> acc(nt, 0.0);
    for (int r = 0; r < rounds; r++)
      for (size_t j = 0; j < nt; j++) {
        double ms = 0.0;
        if ((rc = timed_passes(s, cands[first[j].second], passes, &ms))) return rc;
        acc[j] += ms;
      }
    size_t b = 0;
    for (size_t j = 0; j < nt; j++) {
      note(cands[first[j].second], acc[j] / rounds, 1);
      if (acc[j] < acc[b]) b = j;
    }
    best = cands[first[b].second];
  }
  if (n_log) *n_log = nl;
  if ((rc = irs_scan_configure(s, best.path, best.tile, best.chunk))) return rc;
  *chosen = best;
  return IRS_OK;
}

int irs_scan_restore(irs_scan* s) {
  if (!s) return set_error(IRS_ERR_INVALID, "scan is NULL");
  for (irs_sharedb* e : s->all) {
    int rc = irs_sharedb_set_pair(e, 0);
    if (!rc) rc = irs_sharedb_set_tile(e, 0);
    if (rc) return rc;
  }
  return IRS_OK;
}

}  // extern "C"
