// Rust binding of include/irisb200.h: the `-sys` layer the reference's server
// actor (iris-mpc-gpu/src/server/actor.rs) would link against, e.g. as
// iris-mpc-gpu/src/b200/sys.rs.  One `extern` declaration per function of the
// C header (C `size_t` = `usize`, an array parameter = a pointer to its first
// element, CUDA streams and events as `*mut c_void`).  Rust is not installed
// where this library is built, so this file is not compiled here;
// tests/test_abi_and_harness.py checks that it declares exactly the header's
// functions.
use std::ffi::{c_char, c_int, c_void, CStr};

#[repr(C)] pub struct IrsDeviceManager { _p: [u8; 0] }
#[repr(C)] pub struct IrsShareDb { _p: [u8; 0] }
#[repr(C)] pub struct IrsCircuits { _p: [u8; 0] }
#[repr(C)] pub struct IrsDistanceComparator { _p: [u8; 0] }
#[repr(C)] pub struct IrsGraph { _p: [u8; 0] }
#[repr(C)] pub struct IrsScan { _p: [u8; 0] }
#[repr(C)] #[derive(Clone, Copy)]
pub struct IrsQuerySlot { pub src: u32, pub rot_lo: u32, pub n_rot: u32, pub query: u32 }
pub const IRS_SCAN_SPLIT: i32 = 0;
pub const IRS_SCAN_PAIR: i32 = 1;
pub const IRS_SCAN_FUSED: i32 = 2;
#[repr(C)] #[derive(Clone, Copy)]
pub struct IrsScanCandidate { pub path: i32, pub tile: i32, pub chunk: u64 }
#[repr(C)] #[derive(Clone, Copy)]
pub struct IrsScanTiming { pub cand: IrsScanCandidate, pub ms: f64, pub finalist: i32, pub reserved: i32 }

#[link(name = "irisb200")]
extern "C" {
    pub fn irs_last_error() -> *const c_char;
    pub fn irs_version() -> *const c_char;
    pub fn irs_device_manager_init(device: c_int, out: *mut *mut IrsDeviceManager) -> c_int;
    pub fn irs_device_manager_destroy(dm: *mut IrsDeviceManager) -> c_int;
    pub fn irs_device_manager_stream(dm: *mut IrsDeviceManager, party: c_int,
        stream: *mut *mut c_void) -> c_int;
    pub fn irs_device_manager_synchronize(dm: *mut IrsDeviceManager) -> c_int;
    pub fn irs_device_manager_error(dm: *mut IrsDeviceManager, code: *mut c_int) -> c_int;
    pub fn irs_device_manager_clear_error(dm: *mut IrsDeviceManager) -> c_int;
    pub fn irs_device_manager_test_stall_next_dot(dm: *mut IrsDeviceManager, wait_limit_ns: u64) -> c_int;
    pub fn irs_device_manager_set_batch_counter(dm: *mut IrsDeviceManager, batch_id: u64,
        stream: *mut c_void) -> c_int;
    pub fn irs_device_manager_advance_batch_counter(dm: *mut IrsDeviceManager, stream: *mut c_void) -> c_int;
    pub fn irs_device_manager_set_timing(dm: *mut IrsDeviceManager, on: c_int) -> c_int;
    pub fn irs_device_manager_timings(dm: *mut IrsDeviceManager, buf: *mut c_char, cap: usize,
        reset: c_int) -> c_int;
    pub fn irs_device_manager_get_batch_counter(dm: *mut IrsDeviceManager, batch_id: *mut u64) -> c_int;
    pub fn irs_device_manager_sm_count(dm: *mut IrsDeviceManager, n: *mut c_int) -> c_int;
    pub fn irs_device_manager_set_host_sync(dm: *mut IrsDeviceManager, on: c_int) -> c_int;
    pub fn irs_event_create(ev: *mut *mut c_void) -> c_int;
    pub fn irs_event_record(ev: *mut c_void, stream: *mut c_void) -> c_int;
    pub fn irs_event_synchronize(ev: *mut c_void) -> c_int;
    pub fn irs_event_query(ev: *mut c_void, done: *mut c_int) -> c_int;
    pub fn irs_event_destroy(ev: *mut c_void) -> c_int;
    pub fn irs_device_manager_mem_info(dm: *mut IrsDeviceManager, free_bytes: *mut usize,
        total_bytes: *mut usize) -> c_int;
    pub fn irs_device_alloc(dm: *mut IrsDeviceManager, bytes: usize, ptr: *mut *mut c_void) -> c_int;
    pub fn irs_host_alloc_pinned(bytes: usize, ptr: *mut *mut c_void) -> c_int;
    pub fn irs_host_free_pinned(ptr: *mut c_void) -> c_int;
    pub fn irs_device_free(dm: *mut IrsDeviceManager, ptr: *mut c_void) -> c_int;
    pub fn irs_copy_h2d(dst: *mut c_void, src: *const c_void, bytes: usize, stream: *mut c_void) -> c_int;
    pub fn irs_copy_d2h(dst: *mut c_void, src: *const c_void, bytes: usize, stream: *mut c_void) -> c_int;
    pub fn irs_stream_synchronize(stream: *mut c_void) -> c_int;
    pub fn irs_sharedb_init(dm: *mut IrsDeviceManager, peer_id: c_int, max_db_length: usize,
        query_length: usize, code_length: usize, seed0: *const u32, seed1: *const u32,
        is_remote: c_int, out: *mut *mut IrsShareDb) -> c_int;
    pub fn irs_sharedb_destroy(db: *mut IrsShareDb) -> c_int;
    pub fn irs_sharedb_alloc_db(db: *mut IrsShareDb, max_db_length: usize) -> c_int;
    pub fn irs_sharedb_load_records(db: *mut IrsShareDb, first: usize, n: usize, records: *const u16) -> c_int;
    pub fn irs_sharedb_load_records_i8(db: *mut IrsShareDb, first: usize, n: usize,
        limb0: *const u8, limb1: *const u8) -> c_int;
    pub fn irs_sharedb_fetch_records(db: *mut IrsShareDb, first: usize, n: usize, records: *mut u16) -> c_int;
    pub fn irs_sharedb_set_db_len(db: *mut IrsShareDb, len: usize) -> c_int;
    pub fn irs_sharedb_db_len(db: *mut IrsShareDb, len: *mut usize) -> c_int;
    pub fn irs_sharedb_synth_db(code_engines: *const *mut IrsShareDb,
        mask_engines: *const *mut IrsShareDb, seed: u64, first: usize, n: usize) -> c_int;
    pub fn irs_sharedb_fill_random(db: *mut IrsShareDb, seed: u64, n: usize) -> c_int;
    pub fn irs_device_fill_random(ptr: *mut c_void, bytes: usize, seed: u64, stream: *mut c_void) -> c_int;
    pub fn irs_preprocess_query_share(party: c_int, coefs: *mut u16, n: usize) -> c_int;
    pub fn irs_encode_iris(code_bits: *const u64, mask_bits: *const u64, seed: u64,
        preprocess: c_int, code_out: *mut u16, mask_out: *mut u16) -> c_int;
    pub fn irs_synth_queries(db_seed: u64, q_seed: u64, n_queries: usize,
        planted_entry: *const i64, planted_rot: *const i32, preprocess: c_int, code_out: *mut u16,
        mask_out: *mut u16) -> c_int;
    pub fn irs_sharedb_query_upload(db: *mut IrsShareDb, rows: *const u16, n_rows: usize) -> c_int;
    pub fn irs_sharedb_query_upload_slots(db: *mut IrsShareDb, base: *const u16, n_base: usize,
        slots: *const IrsQuerySlot, n_slots: usize) -> c_int;
    pub fn irs_sharedb_query_upload_rows(db: *mut IrsShareDb, base: *const u16, n_base: usize,
        row_desc: *const u32, n_rows: usize) -> c_int;
    pub fn irs_sharedb_query_put_base(db: *mut IrsShareDb, first: usize, n: usize, base: *const u16) -> c_int;
    pub fn irs_sharedb_query_expand_rows(db: *mut IrsShareDb, n_base: usize, row_desc: *const u32,
        n_rows: usize) -> c_int;
    pub fn irs_sharedb_gather_records(dst: *mut IrsShareDb, src: *mut IrsShareDb, ids: *const u32,
        n: usize) -> c_int;
    pub fn irs_mirror_query_share(coefs: *mut u16, n: usize, flip_imaginary: c_int) -> c_int;
    pub fn irs_sharedb_set_tile(db: *mut IrsShareDb, block_n: c_int) -> c_int;
    pub fn irs_sharedb_set_pair(db: *mut IrsShareDb, on: c_int) -> c_int;
    pub fn irs_sharedb_use_batch_counter(db: *mut IrsShareDb, on: c_int) -> c_int;
    pub fn irs_sharedb_set_batch(db: *mut IrsShareDb, batch_id: u64) -> c_int;
    pub fn irs_sharedb_dot(db: *mut IrsShareDb, offset: usize, len: usize, multiplier: u16,
        stream: *mut c_void) -> c_int;
    pub fn irs_sharedb_dot_many(engines: *const *mut IrsShareDb, multipliers: *const u16, n: c_int,
        offset: usize, len: usize, stream: *mut c_void) -> c_int;
    pub fn irs_sharedb_fetch_results(db: *mut IrsShareDb, host: *mut u16, len: usize) -> c_int;
    pub fn irs_sharedb_result_view(db: *mut IrsShareDb, dev: *mut *const u16, row_stride: *mut usize) -> c_int;
    pub fn irs_circuits_new(dm: *mut IrsDeviceManager, seeds: *const [[u32; 8]; 2],
        out: *mut *mut IrsCircuits) -> c_int;
    pub fn irs_circuits_destroy(c: *mut IrsCircuits) -> c_int;
    pub fn irs_circuits_set_batch(c: *mut IrsCircuits, batch_id: u64) -> c_int;
    pub fn irs_circuits_use_batch_counter(c: *mut IrsCircuits, on: c_int) -> c_int;
    pub fn irs_circuits_compare_threshold_masked_many(c: *mut IrsCircuits,
        code_a: *const *const u16, mask_a: *const *const u16, n: usize, threshold_a: u32,
        res_a: *const *mut u64, res_b: *const *mut u64, opened: *mut u64, stream: *mut c_void) -> c_int;
    pub fn irs_circuits_compare_threshold_masked_many_noalloc(c: *mut IrsCircuits,
        code_a: *const *const u16, mask_a: *const *const u16, n: usize, threshold_a: u32,
        res_a: *const *mut u64, res_b: *const *mut u64, opened: *mut u64, stream: *mut c_void) -> c_int;
    pub fn irs_circuits_extract_msb_of_code(c: *mut IrsCircuits, code_a: *const *const u16,
        n: usize, res_a: *const *mut u64, res_b: *const *mut u64, opened: *mut u64,
        stream: *mut c_void) -> c_int;
    pub fn irs_circuits_or_reduce(c: *mut IrsCircuits, res_a: *const *const u64, n: usize,
        out: *mut u32, stream: *mut c_void) -> c_int;
    pub fn irs_circuits_compare_threshold_masked_many_with_or_tree(c: *mut IrsCircuits,
        code_a: *const *const u16, mask_a: *const *const u16, n: usize, threshold_a: u32,
        out: *mut u32, stream: *mut c_void) -> c_int;
    pub fn irs_circuits_lift_mpc(c: *mut IrsCircuits, mask_a: *const *const u16, n: usize,
        corr: *const *mut u16, stream: *mut c_void) -> c_int;
    pub fn irs_dc_init(dm: *mut IrsDeviceManager, max_queries: usize, max_db_length: usize,
        match_list_cap: usize, out: *mut *mut IrsDistanceComparator) -> c_int;
    pub fn irs_dc_destroy(dc: *mut IrsDistanceComparator) -> c_int;
    pub fn irs_dc_reset(dc: *mut IrsDistanceComparator, stream: *mut c_void) -> c_int;
    pub fn irs_dc_compare_threshold_open(dc: *mut IrsDistanceComparator, c: *mut IrsCircuits,
        code_engines: *const *mut IrsShareDb, mask_engines: *const *mut IrsShareDb, offset: usize,
        len: usize, n_slots: usize, slot_valid: *const u32, slot_query: *const u32,
        threshold_a: u32, self_check: c_int, stream: *mut c_void) -> c_int;
    pub fn irs_dc_set_segments(dc: *mut IrsDistanceComparator, n_slots: usize,
        seg_start: *const u32, seg_query: *const u32, seg_mask: *const u32) -> c_int;
    pub fn irs_dc_compare_threshold_open_prepared(dc: *mut IrsDistanceComparator,
        c: *mut IrsCircuits, code_engines: *const *mut IrsShareDb,
        mask_engines: *const *mut IrsShareDb, offset: usize, len: usize, threshold_a: u32,
        self_check: c_int, stream: *mut c_void) -> c_int;
    pub fn irs_dc_scan_fused(dc: *mut IrsDistanceComparator, c: *mut IrsCircuits,
        code_engines: *const *mut IrsShareDb, mask_engines: *const *mut IrsShareDb, offset: usize,
        len: usize, n_slots: usize, threshold_a: u32, use_segments: c_int, stream: *mut c_void) -> c_int;
    pub fn irs_scan_init(dm: *mut IrsDeviceManager, dc: *mut IrsDistanceComparator, c: *mut IrsCircuits,
        code_engines: *const *mut IrsShareDb, mask_engines: *const *mut IrsShareDb, n_slots: usize,
        db_len: usize, threshold_a: u32, out: *mut *mut IrsScan) -> c_int;
    pub fn irs_scan_destroy(s: *mut IrsScan) -> c_int;
    pub fn irs_scan_candidates(s: *mut IrsScan, out: *mut IrsScanCandidate, cap: usize, n: *mut usize) -> c_int;
    pub fn irs_scan_set_rows(s: *mut IrsScan, n_rows: usize, use_segments: c_int) -> c_int;
    pub fn irs_scan_configure(s: *mut IrsScan, path: c_int, tile: c_int, chunk: usize) -> c_int;
    pub fn irs_scan_current(s: *mut IrsScan, cand: *mut IrsScanCandidate) -> c_int;
    pub fn irs_scan_run(s: *mut IrsScan, stream: *mut c_void) -> c_int;
    pub fn irs_scan_set_timing(s: *mut IrsScan, max_passes: usize) -> c_int;
    pub fn irs_scan_timings(s: *mut IrsScan, gemm_ms: *mut f64, threshold_ms: *mut f64, pass_ms: *mut f64,
        cap: usize, n: *mut usize, reset: c_int) -> c_int;
    pub fn irs_scan_tune(s: *mut IrsScan, passes: c_int, finalists: c_int, rounds: c_int, only_path: c_int,
        chosen: *mut IrsScanCandidate, log: *mut IrsScanTiming, log_cap: usize, n_log: *mut usize) -> c_int;
    pub fn irs_scan_restore(s: *mut IrsScan) -> c_int;
    pub fn irs_dc_take_rows(dc: *mut IrsDistanceComparator, rows: *const u32, n: usize,
        db_len: usize, clear: c_int, counts: *mut u32, ids: *mut u32) -> c_int;
    pub fn irs_dc_enable_distance_capture(dc: *mut IrsDistanceComparator, cap: usize) -> c_int;
    pub fn irs_dc_set_forced_distances(dc: *mut IrsDistanceComparator, query: *const u32,
        entry: *const u32, n: usize) -> c_int;
    pub fn irs_dc_fetch_distances(dc: *mut IrsDistanceComparator, cap: usize, entry: *mut u32,
        row: *mut u32, code: *mut u16, mask: *mut u16, n: *mut usize, reset: c_int) -> c_int;
    pub fn irs_dc_clear_rows(dc: *mut IrsDistanceComparator, first: usize, n: usize,
        stream: *mut c_void) -> c_int;
    pub fn irs_dc_fetch_rows(dc: *mut IrsDistanceComparator, first: usize, n: usize,
        host: *mut u32, cap_words: usize, row_words: *mut usize) -> c_int;
    pub fn irs_dc_fetch_bitmap(dc: *mut IrsDistanceComparator, n_queries: usize, db_len: usize,
        host: *mut u64) -> c_int;
    pub fn irs_dc_fetch_matches(dc: *mut IrsDistanceComparator, pairs: *mut u32, cap: usize,
        n: *mut usize) -> c_int;
    pub fn irs_dc_get_partial_results(dc: *mut IrsDistanceComparator, n_queries: usize,
        db_len: usize, ids: *mut u32, cap: usize, n: *mut usize) -> c_int;
    pub fn irs_dc_join_db_matches(dc: *mut IrsDistanceComparator,
        right: *mut IrsDistanceComparator, or_policy: *const u32, n_queries: usize, db_len: usize,
        stream: *mut c_void) -> c_int;
    pub fn irs_dc_join_batch_matches(dc: *mut IrsDistanceComparator,
        right: *mut IrsDistanceComparator, n_queries: usize, stream: *mut c_void) -> c_int;
    pub fn irs_dc_fetch_final_results(dc: *mut IrsDistanceComparator, n_queries: usize,
        final_results: *mut u32, match_counters: *mut u32, all_matches: *mut u32) -> c_int;
    pub fn irs_graph_begin_capture(dm: *mut IrsDeviceManager) -> c_int;
    pub fn irs_graph_end_capture(dm: *mut IrsDeviceManager, out: *mut *mut IrsGraph) -> c_int;
    pub fn irs_graph_launch(g: *mut IrsGraph, stream: *mut c_void) -> c_int;
    pub fn irs_graph_destroy(g: *mut IrsGraph) -> c_int;
}

pub fn check(rc: c_int) -> eyre::Result<()> {
    if rc == 0 { return Ok(()); }
    let msg = unsafe { CStr::from_ptr(irs_last_error()) }.to_string_lossy().into_owned();
    Err(eyre::eyre!("irisb200 error {rc}: {msg}"))
}
