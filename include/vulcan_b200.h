/* vulcan_b200.h -- C ABI of libvulcan_b200.so, the sm_100a DDA search hot path.
 *
 * Conventions
 *   - Every pointer argument is a DEVICE pointer unless its comment says "host".
 *   - `stream` is a cudaStream_t passed as void*; launches are asynchronous on it.
 *   - Every function returns 0 on success, a cudaError_t code (> 0) if a launch failed, or a negative VK_E_* code
 *     for a rejected argument.  Nothing allocates device memory unless its comment says so: the caller sizes every
 *     buffer (the *_count / *_plan calls report the sizes).
 *   - No hidden global state except the process-wide constants of the reference-compatible entry points
 *     (vk_set_params / vk_set_nterm / vk_set_tol_da, per device, as in the reference).  The B200 entry points take
 *     their fragment constants by value (vk_frag_params), so threads with their own streams can call them
 *     concurrently.
 *
 * Part 1 keeps the reference's exported names and argument lists (vulcan/gpu/_lib.py:22-35 binds them with
 * ctypes), so the reference's own engine can load this library unchanged.  Part 2 is the B200 layout: a tiled
 * fragment index (row tiles, postings sorted by exact f32 fragment m/z, per-tile CSR over integer coarse m/z bins)
 * and the device stages of the search.
 */
#ifndef VULCAN_B200_H
#define VULCAN_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VK_E_ARG (-1)       /* invalid argument (size, alignment, layout limit) */
#define VK_E_CAPACITY (-2)  /* an output buffer is too small; the needed size was written where documented */
#define VK_E_TOO_LARGE (-3) /* the input is larger than a fixed-size internal buffer allows */

/* ============================================================ Part 1: reference-compatible entry points */

/* Replaces vulcan/gpu/kernels.cu:381-385: Sage f32 residue masses (26, by letter), static and variable
 * modification deltas (26 each); host pointers; copied to this device's constant memory. */
int vk_set_params(const float* mono, const float* stat, const float* var);
/* Replaces kernels.cu:387: variable peptide-N-term delta (mask bit 63). */
int vk_set_nterm(float nterm);
/* Replaces kernels.cu:389: fragment tolerance unit, 0 = ppm, 1 = Da. */
int vk_set_tol_da(int da);

/* Replaces kernels.cu:391-399 (frag_count_kernel): index fragments per row (ion index > min_ion_index and
 * fmin <= neutral fragment mass <= fmax). */
int vk_frag_count(int64_t n, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                  const uint8_t* res, int min_ion_index, float fmin, float fmax, int32_t* count, void* stream);
/* Replaces kernels.cu:401-411 (frag_emit_kernel): int64 keys chunk<<50 | logbin<<32 | local<<16 | fine. */
int vk_frag_emit(int64_t n, const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                 const uint8_t* res, int min_ion_index, float fmin, float fmax, double inv_logw, int chunk_size,
                 int64_t row0, const int64_t* out_off, int64_t* keys, void* stream);
/* Replaces kernels.cu:413-431 (k1_kernel): K1 counts over the reference's (chunk, log bin) CSR; appends
 * (hyp, row, count) for count >= thr at atomicAdd(n_out) (entries beyond cap are dropped, n_out still counts them);
 * hyp_scored / hyp_matched accumulate. */
int vk_k1(int n_items, const int32_t* it_hyp, const int32_t* it_chunk, const int32_t* it_lo, const int32_t* it_hi,
          const int32_t* hyp_spec, const int8_t* hyp_maxfz, const int64_t* pk_off, const float* pk_mass,
          const uint32_t* offsets, const uint32_t* entries, int n_bins, int chunk0, int chunk_size, int tile,
          float tol_lo, float tol_hi, float fmin, double inv_logw, int thr, int64_t cap,
          unsigned long long* n_out, int32_t* out_hyp, int32_t* out_row, int32_t* out_cnt,
          unsigned int* hyp_scored, unsigned long long* hyp_matched, void* stream);
/* Replaces kernels.cu:433-445 (k1_brute_kernel): brute-force K1 count of each (hyp, row) pair. */
int vk_k1_brute(int64_t n, const int32_t* c_hyp, const int32_t* c_row, const int32_t* hyp_spec,
                const int8_t* hyp_maxfz, const int64_t* pk_off, const float* pk_mass, const int64_t* seq_off,
                const uint8_t* len, const uint64_t* mask, const float* mass32, const uint8_t* res,
                int min_ion_index, float fmin, float fmax, float tol_lo, float tol_hi, double inv_logw,
                int32_t* out_cnt, void* stream);
/* Replaces kernels.cu:447-458 (k2_kernel, closed mode): exact b/y rescoring of candidates grouped by spectrum
 * (cand_off[n_spec+1]); spectrum bs uses peaks of spec_ids[bs] (first 512 mass-sorted peaks).  `threads` is
 * accepted for signature compatibility; the launch shape is chosen here. */
int vk_k2(int n_spec, const int64_t* cand_off, const int32_t* c_row, const int8_t* c_maxfz, const int32_t* spec_ids,
          const int64_t* pk_off, const float* pk_mass, const float* pk_int, const int64_t* seq_off,
          const uint8_t* len, const uint64_t* mask, const float* mass32, const uint8_t* res, float tol_lo,
          float tol_hi, double* o_hs, float* o_sb, float* o_sy, float* o_ppm, int16_t* o_mb, int16_t* o_my,
          int16_t* o_lb, int16_t* o_ly, int threads, void* stream);
/* Replaces kernels.cu:461-472: K2 with a per-candidate precursor delta (shifted + unshifted ions, best site). */
int vk_k2_shift(int n_spec, const int64_t* cand_off, const int32_t* c_row, const int8_t* c_maxfz,
                const int32_t* spec_ids, const int64_t* pk_off, const float* pk_mass, const float* pk_int,
                const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                const uint8_t* res, float tol_lo, float tol_hi, const float* c_shift, double* o_hs, float* o_sb,
                float* o_sy, float* o_ppm, int16_t* o_mb, int16_t* o_my, int16_t* o_lb, int16_t* o_ly,
                int threads, void* stream);

/* ============================================================ Part 2: B200 layout and device stages */

/* Fragment constants by value (what vk_set_params/vk_set_nterm/vk_set_tol_da hold globally in Part 1). */
typedef struct {
  float mono[26];
  float stat[26];
  float var[26];
  float nterm;
  int tol_da;
} vk_frag_params;

/* Tiled fragment index.  Rows (mass-sorted peptidoforms) are cut into tiles of tile_rows = 2^tile_shift rows.
 * A fragment's key is f32bits(fragment) - f32bits(fmin), mass_bits = bit length of f32bits(fmax) - f32bits(fmin)
 * wide; a tile's fragments are sorted by (key, row), i.e. by exact f32 mass, then row.  The coarse m/z bin of a
 * fragment is the top cbin_bits bits of its key (an integer bin in f32-bit space); cbin_off[tile*stride + b]
 * (u16, relative to the tile's first posting; stride = 2^cbin_bits + 1 rounded up to 8) is the CSR over those
 * bins.  The bin being implicit in the position, a posting is one u32 holding the rest of the key and the local
 * row: (key mod 2^(mass_bits - cbin_bits)) << row_bits | (row - tile*tile_rows), row_bits = 32 - mass_bits +
 * cbin_bits.  tile_off[n_tiles+1] (i64) locates each tile's postings (16-byte aligned, padding 0xffffffff after
 * the last bin).  bitmap (u32, 16-byte aligned; vk_tindex_bitmap, vk_tindex_bitmap_bytes): each tile's presence
 * bitmap, 2^B bits per coarse bin (B = 6 in this build), the words of tile t's bin b at (t * 2^cbin_bits + b) *
 * 2^B / 32; bit s of bin b is set when a posting of bin b has (low key bits) >> (low_bits - B) == s (low_bits =
 * mass_bits - cbin_bits; with low_bits < B the low key itself); K1 drops the tolerance windows whose bits are all
 * clear. */
typedef struct {
  int64_t n_rows;
  int64_t n_tiles;
  int64_t n_postings;
  int32_t tile_shift;       /* log2(tile_rows) */
  int32_t row_bits;
  int32_t mass_bits;
  int32_t cbin_bits;        /* coarse bins per tile = 2^cbin_bits */
  uint32_t fmin_bits;
  uint32_t fmax_bits;
  int32_t min_ion_index;
  int32_t max_tile_postings;
  const int64_t* tile_off;
  const uint16_t* cbin_off;
  const uint32_t* postings;
  const uint32_t* bitmap;
} vk_tindex;

/* Layout of a tiled index for tile_rows/fmin/fmax: fills tile_shift, row_bits, mass_bits, cbin_bits, fmin_bits,
 * fmax_bits, n_tiles (host struct).  VK_E_ARG if tile_rows is not a power of two in [32, 1024] or does not fit
 * row_bits, or cbin_bits is outside [1, min(12, mass_bits - 1)]. */
int vk_tindex_layout(int64_t n_rows, int tile_rows, float fmin, float fmax, int min_ion_index, int cbin_bits,
                     vk_tindex* ix);
/* Postings per tile: tile_count[n_tiles] (i64) from the peptidoform table. */
int vk_tindex_count(const vk_tindex* ix, const vk_frag_params* fp, const int64_t* seq_off, const uint8_t* len,
                    const uint64_t* mask, const float* mass32, const uint8_t* res, int64_t* tile_count,
                    void* stream);
/* Fill postings and cbin_off of a tiled index whose tile_off (exclusive scan of tile_count) is in place.
 * max_tile_postings (host, from tile_count) sizes the per-tile sort; VK_E_TOO_LARGE above 16384. */
int vk_tindex_emit(const vk_tindex* ix, const vk_frag_params* fp, const int64_t* seq_off, const uint8_t* len,
                   const uint64_t* mask, const float* mass32, const uint8_t* res, uint32_t* postings,
                   uint16_t* cbin_off, void* stream);
/* Presence bitmaps of every tile (ix->tile_off, cbin_off and postings in place) into bitmap (u32, 16-byte aligned,
 * vk_tindex_bitmap_bytes(ix) bytes), see vk_tindex. */
int vk_tindex_bitmap(const vk_tindex* ix, uint32_t* bitmap, void* stream);
int64_t vk_tindex_bitmap_bytes(const vk_tindex* ix);

/* Exclusive scan of n int64 values: out[0] = 0, out[i+1] = sum(in[0..i]) (out has n+1 entries; in == out+1
 * is allowed).  Uses `tmp` of vk_scan_tmp_bytes(n) bytes.  vk_scan_kernels(n) = the kernels one scan of n values
 * launches: 1 up to 4,096 values, 2 up to 8,388,608 (block sums, then each block adds the sums before it), 3
 * beyond (the block sums scanned by a kernel of their own); n == 0 launches none (a memset). */
int64_t vk_scan_tmp_bytes(int64_t n);
int vk_scan_i64(const int64_t* in, int64_t n, int64_t* out, void* tmp, void* stream);
int vk_scan_kernels(int64_t n);

/* The same exclusive scan without the caller's scratch buffer; it allocates nothing.  No counterpart in the
 * reference.  For callers that cannot allocate device memory on this path: a foreign-language binding (cgo, JNI,
 * plain C) that holds only the input and output buffers and has no device allocator to hand out scratch, or a
 * stage thread that must not call cudaMalloc / cudaFree because they synchronise the whole device and would stall
 * the other streams' searches.
 *   - Scratch: the block partial sums live in one fixed device array inside the library (64 KiB on every device
 *     that loads it, held until the process exits).  n may be at most vk_scan_noalloc_max_n() = 33,554,432;
 *     larger n returns VK_E_TOO_LARGE and launches nothing.
 *   - Set-up: the first call with n > 0 on a device looks up the array's device address (cudaGetSymbolAddress)
 *     with that device current and keeps it for the life of the process; make that first call before any stream
 *     capture (n == 0 looks nothing up).  The kept address does not survive a cudaDeviceReset of that device in
 *     the same process: after a reset, do not call this entry point on that device again.
 *   - Sharing: every call on a device uses the same array.  Calls whose kernels may overlap on the GPU (other
 *     streams, other host threads) race on it and give wrong sums; order them (one stream, or events).
 *     Nothing in the array has to start at zero; each call overwrites what it reads. */
int64_t vk_scan_noalloc_max_n(void);
int vk_scan_i64_noalloc(const int64_t* in, int64_t n, int64_t* out, void* stream);

/* K0 peak view (reference vulcan/gpu/engine.py:171-210), two calls: vk_k0_count writes kept[n_spec] (i64) =
 * min(#peaks with fmin <= mz <= fmax and not NaN, max_peaks), easy[n_spec] (u8: 1 = the raw peaks are already in
 * (mass asc, intensity desc) order, no NaN, at most max_peaks in range; 2 = in that order with more in range and
 * at most 512 raw peaks; 3 = the same with more raw peaks; 0 = otherwise) and the indices of the code 0 and 3
 * spectra into hard_list[n_spec] (i32, any order) with their number in *n_hard (device i32, zeroed by the call);
 * after the caller's scan of kept into pk_off[n_spec+1], vk_k0_fill writes mass-sorted peaks (mass = mz - PROTON)
 * of the top max_peaks by (intensity desc, mass desc), tic[n_spec] (f32 of the f64 sum) and valid[n_spec] (u8,
 * kept >= min_peaks): code 1 by a stream copy, code 2 by a warp each and code 3 by a CTA each (radix selection of
 * the kept peaks, compaction in input order), code 0 (unsorted or NaN m/z) by shared-memory sorts.  max_raw
 * (host) = the largest
 * raw peak count of a spectrum, at most 16384 (one CTA sorts a spectrum in shared memory). */
int vk_k0_count(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                float fmax, int max_peaks, int64_t* kept, uint8_t* easy, int32_t* hard_list, int32_t* n_hard,
                void* stream);
int vk_k0_fill(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
               float fmax, int max_peaks, int min_peaks, const int64_t* pk_off, float* pk_mass, float* pk_int,
               float* tic, uint8_t* valid, int max_raw, const uint8_t* easy, const int32_t* hard_list,
               const int32_t* n_hard, void* stream);
/* vk_k0_fill in two halves with its arguments: vk_k0_fill_easy writes the code 1 and 2 spectra, vk_k0_fill_hard the
 * code 0 and 3 spectra.  They write disjoint outputs, so a caller may run them on two streams (both after
 * vk_k0_count and the scan); vk_k0_fill runs one after the other. */
int vk_k0_fill_easy(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                    float fmax, int max_peaks, int min_peaks, const int64_t* pk_off, float* pk_mass, float* pk_int,
                    float* tic, uint8_t* valid, int max_raw, const uint8_t* easy, const int32_t* hard_list,
                    const int32_t* n_hard, void* stream);
int vk_k0_fill_hard(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                    float fmax, int max_peaks, int min_peaks, const int64_t* pk_off, float* pk_mass, float* pk_int,
                    float* tic, uint8_t* valid, int max_raw, const uint8_t* easy, const int32_t* hard_list,
                    const int32_t* n_hard, void* stream);

/* K0 peak view in the window peak mode (reference vulcan/gpu/engine.py:182-183, peak_mode "window"), the same two
 * calls and buffers: the top window_k peaks (intensity desc, mass desc) of every window w = floor(mz * (1.0f /
 * window_th)) (f32, the reference's division of an f32 CUDA tensor by a Python float) of the in-range peaks, then
 * mass ascending (equal masses: window ascending, then intensity descending); no cap on the total.  kept[s] =
 * sum over windows of min(count, window_k); easy[s]: 1 = already in that order with no window over window_k (a
 * copy), 2 = in that order, some window over window_k, none over 128 peaks (a warp), 0 = otherwise (hard_list, a
 * CTA sort).  VK_E_ARG unless window_th > 0 and 0 <= floor(fmin / window_th), floor(fmax / window_th) <= 999 (the
 * reference's group id spectrum * 1000 + window lets windows of neighbouring spectra merge beyond that). */
int vk_k0w_count(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                 float fmax, float window_th, int window_k, int64_t* kept, uint8_t* easy, int32_t* hard_list,
                 int32_t* n_hard, void* stream);
int vk_k0w_fill(int n_spec, const int64_t* raw_off, const float* raw_mz, const float* raw_int, float fmin,
                float fmax, float window_th, int window_k, int min_peaks, const int64_t* pk_off, float* pk_mass,
                float* pk_int, float* tic, uint8_t* valid, int max_raw, const uint8_t* easy,
                const int32_t* hard_list, const int32_t* n_hard, void* stream);

/* Hypotheses (reference vulcan/gpu/host.py:64-91), two calls like K0: vk_hyp_count writes n_hyp[n_spec] (i64);
 * vk_hyp_fill writes, at hyp_off[s], the spectrum's hypotheses in (charge, isotope) order with f32 Sage
 * arithmetic and the row window [lo, hi) by binary search of the mass-sorted index masses (hyp_off: the scan of
 * n_hyp, n_spec + 1 entries; the searches of all hyp_off[n_spec] hypotheses run in parallel, a thread per bound). */
int vk_hyp_count(int n_spec, const uint8_t* valid, const double* precursor_mz, const int8_t* charge, int z_lo,
                 int z_hi, int iso_lo, int iso_hi, int64_t* n_hyp, void* stream);
int vk_hyp_fill(int n_spec, const uint8_t* valid, const double* precursor_mz, const int8_t* charge, int z_lo,
                int z_hi, int iso_lo, int iso_hi, float ppm_lo, float ppm_hi, int max_fragment_charge,
                const float* idx_mass32, int64_t n_rows, const int64_t* hyp_off, int32_t* h_spec, int8_t* h_z,
                int8_t* h_iso, float* h_pm, float* h_M, int64_t* h_lo, int64_t* h_hi, int8_t* h_maxfz,
                void* stream);

/* K1 on the tiled index.  Work items are (tile, hypothesis) pairs grouped by tile:
 *   vk_k1_plan_count: items per tile (tile_items[n_tiles], i64, zeroed by the call) and window sizes
 *                     (win_len[n_hyp], i64);
 *   vk_k1_plan_fill:  with tile_item_off (scan of tile_items) in place, writes item_hyp[n_items] (i32) grouped by
 *                     tile (order inside a tile is unspecified; results do not depend on it);  `cursor` is an
 *                     n_tiles i64 scratch;
 *   vk_k1_tiles:      dense counts cnt[win_off[h] + row - lo[h]] (i32) for every window row of every hypothesis.
 * Counts equal the reference's brute force (kernels.cu:195-232): #(peak p, fragment charge z < maxfz, index
 * fragment f) with tol_bound(p*z, tol_lo) <= f <= tol_bound(p*z, tol_hi) in f32.  `status` (device i32, zeroed by
 * the caller) gets VK_STATUS_WAIT_TIMEOUT if a tile copy did not complete within the bounded wait.  `warps` (1..16)
 * per CTA, one CTA per tile with work.  isum (may be
 * NULL; then pk_int and tic may be NULL too): per window row the summed intensity of its matches, u32 fixed point
 * = sum of round(intensity * 2^24 / tic[s]), for the candidate pruner's features.  VK_E_TOO_LARGE if a tile and
 * the histograms do not fit one CTA's shared memory.
 * The buffers may be sized by bounds instead of the exact totals (no host read-back between the calls):
 * item_hyp holds item_cap entries, cnt / isum cnt_cap; items or windows that would not fit are skipped and set
 * VK_STATUS_OVERFLOW in `status` (the caller then retries with larger buffers).
 * The index's tile bitmaps (ix->bitmap) are required.  pk_keys / pk_filt (may be NULL with n_kz = 0): the window
 * keys and filter words of vk_k1_peak_keys for fragment charges 1..n_kz, plane stride kstride (pk_keys 8-byte
 * aligned); higher charges are computed inside the kernel.  The result does not depend on them: they only save
 * recomputing a peak's window for every tile its hypotheses cover.
 *   vk_k1_peak_keys:  keys[(z-1)*kstride + p] = (ka, kb), two u32 per kept peak p < min(*n_peaks, kstride)
 *                     (n_peaks: device i64, e.g. pk_off + n_spec) and charge z = 1..n_kz: the tolerance window of
 *                     mass pk_mass[p]*z as an inclusive key range of the tiled index (key = f32bits - fmin bits),
 *                     clamped to the fragment range; ka > kb when the window misses it.  filt[(z-1)*kstride + p]
 *                     (u32): the window's bitmap position ga (bits 0..19) and span min(gb - ga, 4095) (bits
 *                     20..31), 0xffffffff when the window misses the range. */
int vk_k1_plan_count(const vk_tindex* ix, int64_t n_hyp, const int64_t* h_lo, const int64_t* h_hi,
                     int64_t* tile_items, int64_t* win_len, void* stream);
int vk_k1_plan_fill(const vk_tindex* ix, int64_t n_hyp, const int64_t* h_lo, const int64_t* h_hi,
                    const int64_t* tile_item_off, int64_t* cursor, int32_t* item_hyp, int64_t item_cap,
                    int32_t* status, void* stream);
int vk_k1_tiles(const vk_tindex* ix, const vk_frag_params* fp, float tol_lo, float tol_hi, int warps,
                const int64_t* tile_item_off, const int32_t* item_hyp, int64_t n_hyp, int64_t item_cap,
                const int32_t* h_spec, const int8_t* h_maxfz, const int64_t* h_lo, const int64_t* h_hi,
                const int64_t* win_off, int64_t cnt_cap, const int64_t* pk_off, const float* pk_mass, int32_t* cnt,
                int32_t* status, const float* pk_int, const float* tic, uint32_t* isum, const uint32_t* pk_keys,
                const uint32_t* pk_filt, int n_kz, int64_t kstride, void* stream);
int vk_k1_peak_keys(const vk_tindex* ix, const vk_frag_params* fp, float tol_lo, float tol_hi, const int64_t* n_peaks,
                    const float* pk_mass, int n_kz, int64_t kstride, uint32_t* keys, uint32_t* filt, void* stream);
/* K1 in hit-list form (the learned-pruned search, the open / mass-offset modes): the same counting as vk_k1_tiles,
 * but instead of a dense count per window row, each (tile, hypothesis) item writes the rows of its tile with count >=
 * thr (>= 1; h_thr[h] instead when h_thr is given, i32 per hypothesis) in row order to the start of its segment of
 * the hypothesis' region -- the slots win_off[h] + (row - lo[h]) of the window rows the tile holds -- as hit_rc
 * (u64: count << 32 | row) and, with pk_int/tic, hit_isum (the summed matched intensity of vk_k1_tiles' isum), and
 * their number to seg_cnt (u32, same slots) at the segment's first slot; hyp_shift[h] (i8, zeroed by the caller) gets
 * the tiling's tile_shift, which fixes the segment boundaries; hyp_scored (u32, rows with count > 0) and hyp_matched
 * (u64, sum of counts) are accumulated with atomics (zeroed by the caller).  No atomic decides a position: the
 * layout does not depend on scheduling.  cnt_cap bounds hit_rc / hit_isum like vk_k1_tiles' cnt.  Reference
 * semantics: kernels.cu:170-189 (threshold append, scored, matched). */
int vk_k1_hits(const vk_tindex* ix, const vk_frag_params* fp, float tol_lo, float tol_hi, int warps,
               const int64_t* tile_item_off, const int32_t* item_hyp, int64_t n_hyp, int64_t item_cap,
               const int32_t* h_spec, const int8_t* h_maxfz, const int64_t* h_lo, const int64_t* h_hi,
               const int64_t* win_off, int64_t cnt_cap, const int64_t* pk_off, const float* pk_mass, int thr,
               const int32_t* h_thr, uint64_t* hit_rc, uint32_t* hit_isum, uint32_t* seg_cnt, int8_t* hyp_shift,
               uint32_t* hyp_scored, uint64_t* hyp_matched, int32_t* status, const float* pk_int, const float* tic,
               const uint32_t* pk_keys, const uint32_t* pk_filt, int n_kz, int64_t kstride, void* stream);

/* Top-K + pair closure (reference vulcan/gpu/engine.py:284-312) per spectrum, from the dense K1 counts.
 * Spectrum s owns hypotheses [spec_hyp_off[s], spec_hyp_off[s+1]).  Per spectrum: entries with count >= thr,
 * ranked by (count desc, row desc, hypothesis asc), the first topk kept; with pair_closure their partner rows are
 * added with count -1; duplicates of (spectrum, row) merge to the lowest hypothesis and highest count.  Output
 * slots: spectrum s writes n_cand[s] candidates sorted by row at [s*cap, s*cap + n_cand[s]) of c_hyp (i64),
 * c_row (i64), c_cnt (i64); cap >= (pair_closure ? 2 : 1) * topk.  Also hyp_scored (u32, #rows with count > 0)
 * and hyp_matched (u64, sum of counts) per hypothesis, and their sums per spectrum (spec_scored, spec_matched,
 * i64; may be NULL).  cnt holds cnt_cap entries: a window whose slice would end past it counts as empty. */
int vk_select_topk(int n_spec, const int64_t* spec_hyp_off, const int64_t* h_lo, const int64_t* h_hi,
                   const int64_t* win_off, const int32_t* cnt, int64_t cnt_cap, const int64_t* partner, int thr,
                   int topk, int pair_closure, int cap, int64_t* c_hyp, int64_t* c_row, int64_t* c_cnt, int64_t* n_cand,
                   uint32_t* hyp_scored, uint64_t* hyp_matched, int64_t* spec_scored, int64_t* spec_matched,
                   void* stream);

/* Top-K + pair closure from the hit lists of vk_k1_hits (reference vulcan/gpu/engine.py:284-312): per spectrum
 * its hypotheses' hits ranked by (count desc, row desc, hypothesis asc), the first topk kept (all when fewer);
 * with pair_closure the partner rows added with count -1; sorted by row, duplicate rows merged to the lowest
 * hypothesis and highest count: the slots of vk_select_topk (cap >= (pair_closure ? 2 : 1) * topk) plus c_isum
 * (u32, the kept hit's intensity sum, 0 for a partner-only row; NULL when hit_isum is NULL), and spec_scored /
 * spec_matched (i64, may be NULL) summed from K1's per-hypothesis totals; h_lo / h_hi / win_off / hyp_shift /
 * seg_cnt locate each hypothesis' hit segments (per 32 segments, one parallel read of their counts, then one of
 * their hits).  The same candidates as vk_select_topk over vk_k1_tiles' dense counts with
 * thr = vk_k1_hits' thr.  Without closure, when a spectrum's windows are pairwise disjoint (the usual case), the
 * hits are collected in row order and kept in that order, with no sort. */
int vk_select_hits(int n_spec, const int64_t* spec_hyp_off, const int64_t* h_lo, const int64_t* h_hi,
                   const int64_t* win_off, const int8_t* hyp_shift, const uint32_t* seg_cnt, const uint64_t* hit_rc,
                   const uint32_t* hit_isum,
                   const uint32_t* hyp_scored, const uint64_t* hyp_matched, int topk, int pair_closure,
                   const int64_t* partner, int cap, int64_t* c_hyp, int64_t* c_row, int64_t* c_cnt, uint32_t* c_isum,
                   int64_t* n_cand, int64_t* spec_scored, int64_t* spec_matched, void* stream);

/* Compaction of per-spectrum slots into a flat candidate list: with cand_off = scan(n_cand), copies slot s to
 * [cand_off[s], cand_off[s+1]) and writes c_maxfz from h_maxfz[c_hyp].  vk_compact_hits also carries the
 * intensity sums (s_isum -> c_isum). */
int vk_compact_cands(int n_spec, int cap, const int64_t* n_cand, const int64_t* cand_off, const int64_t* s_hyp,
                     const int64_t* s_row, const int64_t* s_cnt, const int8_t* h_maxfz, int64_t* c_hyp,
                     int64_t* c_row, int64_t* c_cnt, int32_t* c_row32, int8_t* c_maxfz, void* stream);
int vk_compact_hits(int n_spec, int cap, const int64_t* n_cand, const int64_t* cand_off, const int64_t* s_hyp,
                    const int64_t* s_row, const int64_t* s_cnt, const uint32_t* s_isum, const int8_t* h_maxfz,
                    int64_t* c_hyp, int64_t* c_row, int64_t* c_cnt, int32_t* c_row32, int8_t* c_maxfz,
                    uint32_t* c_isum, void* stream);

/* K2 exact rescoring (reference kernels.cu:263-376), B200 launch: one warp per spectrum, lanes over candidates,
 * the spectrum's (first 512) peaks in shared memory.  Candidates of spectrum s are [cand_off[s], cand_off[s+1])
 * (cand_off has n_spec+1 entries, spectrum ids are 0..n_spec-1).  c_shift NULL: the closed mode; else the
 * per-candidate precursor shift (Da, f32) of the open / mass-offset modes: shifted and unshifted ions scored as
 * the reference's shift mode (kernels.cu:294-363). */
int vk_k2_spectra(const vk_frag_params* fp, int n_spec, const int64_t* cand_off, const int32_t* c_row,
                  const int8_t* c_maxfz, const int64_t* pk_off, const float* pk_mass, const float* pk_int,
                  const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                  const uint8_t* res, float tol_lo, float tol_hi, const float* c_shift, double* o_hs, float* o_sb,
                  float* o_sy, float* o_ppm, int16_t* o_mb, int16_t* o_my, int16_t* o_lb, int16_t* o_ly,
                  void* stream);
/* vk_k2_spectra without the shift, one thread per candidate (grid-stride over cand_off[n_spec] candidates, the
 * spectrum found by binary search of cand_off) with the peaks read in global memory: for sparse candidate lists (a
 * few per spectrum, e.g. after the learned pruner), where a warp per spectrum would leave most lanes idle.  Same
 * outputs, bit for bit. */
int vk_k2_cands(const vk_frag_params* fp, int n_spec, const int64_t* cand_off, const int32_t* c_row,
                const int8_t* c_maxfz, const int64_t* pk_off, const float* pk_mass, const float* pk_int,
                const int64_t* seq_off, const uint8_t* len, const uint64_t* mask, const float* mass32,
                const uint8_t* res, float tol_lo, float tol_hi, double* o_hs, float* o_sb, float* o_sy, float* o_ppm,
                int16_t* o_mb, int16_t* o_my, int16_t* o_lb, int16_t* o_ly, void* stream);

/* PSM ranking (reference vulcan/gpu/engine.py:366-392): per spectrum, candidates with matched_b + matched_y >=
 * min_matched ranked by (hyperscore desc, row asc); the first `report` go to slots [s*report, ...): psm_cand (i64,
 * candidate index or -1), psm_rank (i32, 1-based), psm_dnext, psm_dbest (f64).  n_psm[s] = number written. */
int vk_psm_rank(int n_spec, const int64_t* cand_off, const int64_t* c_row, const double* hs, const int16_t* mb,
                const int16_t* my, int min_matched, int report, int64_t* psm_cand, int32_t* psm_rank,
                double* psm_dnext, double* psm_dbest, int32_t* n_psm, void* stream);
/* vk_psm_rank with one thread per spectrum scanning its candidates in order (a warp per spectrum above): for sparse
 * candidate lists (a few per spectrum after the learned pruner), where most of a warp would idle.  Same outputs. */
int vk_psm_rank_sparse(int n_spec, const int64_t* cand_off, const int64_t* c_row, const double* hs, const int16_t* mb,
                       const int16_t* my, int min_matched, int report, int64_t* psm_cand, int32_t* psm_rank,
                       double* psm_dnext, double* psm_dbest, int32_t* n_psm, void* stream);

/* PSM table columns of every ranked slot (the features of the reference's psm_table, vulcan/gpu/engine.py:361-432,
 * computed on the device), packed into one byte buffer for a single device-to-host copy.  Slot j (0 <= j < slots,
 * spectrum j / report) takes candidate psm_cand[j] (-1: empty slot, its row is written with valid = 0 and
 * arbitrary values; every index it reads is clamped into its table).  Column c (VK_PSM_COLS of them, in this
 * order: valid u8, spec_idx i64, rank i32, pf_row i64, pf_id u64, charge i8, isotope_error i8, expmass f32,
 * calcmass f32, delta_mass_ppm f32, hyperscore f64, delta_next f64, delta_best f64, matched_b i16, matched_y i16,
 * matched_peaks i16, summed_intensity f32, matched_intensity_pct f32, average_ppm f32, longest_b i16, longest_y
 * i16, longest_y_pct f32, peptide_len i16, missed_cleavages u8, n_var u8, k1_count i32, scored_candidates i32,
 * poisson f64) holds `slots` elements starting at byte col_off[c] (host array; multiples of 8) of `packed`.
 * Arithmetic: f32 masses and percentages, f64 Poisson term, one rounding per operation in the reference's order.
 * row_pos (may be NULL): the exclusive prefix count of filled slots (slots + 1 entries, e.g. a scan of
 * psm_cand >= 0); with it the filled slots are written contiguously in slot order (slot j to row row_pos[j]),
 * empty slots not at all, and column 0 holds their number row_pos[slots] as one i64 instead of the valid bytes
 * (0 when slots = 0; column 0 then needs 8 bytes), so the host reads plain slices. */
#define VK_PSM_COLS 28
typedef struct {
  const int64_t* psm_cand;
  const int32_t* psm_rank;
  const double* dnext;
  const double* dbest;
  const int64_t* c_hyp;
  const int64_t* c_row;
  const int64_t* c_cnt;
  const int8_t* h_z;
  const int8_t* h_iso;
  const float* h_pm;
  int64_t n_hyp;            /* entries of the hypothesis columns */
  const int64_t* spec_scored;
  const int64_t* spec_matched;
  const float* tic;
  const double* hs;
  const float* sb;
  const float* sy;
  const float* ppm;
  const int16_t* mb;
  const int16_t* my;
  const int16_t* lb;
  const int16_t* ly;
  const float* mass32;
  const uint8_t* length;
  const int64_t* pf_id;
  const uint8_t* missed;
  const uint8_t* n_var;
  int64_t n_rows;           /* index rows */
} vk_psm_pack_in;
int vk_pack_psms(const vk_psm_pack_in* in, int64_t slots, int report, const int64_t* col_off,
                 const int64_t* row_pos, uint8_t* packed, void* stream);

/* ============================================================ Part 3: fused persistent search */

/* Inputs of the fused search.  Spectra are the batch's (global ids 0..n_spec-1, peaks and hypotheses grouped by
 * spectrum as vk_k0_fill / vk_hyp_fill write them); spec_ids (may be NULL) selects the n_work spectra to search. */
typedef struct {
  int n_spec;
  int n_work;
  const int32_t* spec_ids;
  const int64_t* pk_off;
  const float* pk_mass;
  const float* pk_int;
  const int64_t* spec_hyp_off;
  const int64_t* h_lo;
  const int64_t* h_hi;
  const int8_t* h_maxfz;
  const int64_t* partner;
  const int64_t* seq_off;
  const uint8_t* len;
  const uint64_t* mask;
  const float* mass32;
  const uint8_t* res;
  float tol_lo, tol_hi;
  int thr, topk, pair_closure, min_matched, report;
} vk_fused_in;

/* Reported PSMs, slot s*report + k (k < n_psm[s]); row = -1 in unused slots. */
typedef struct {
  int64_t* row;
  int64_t* hyp;
  int64_t* k1;
  int32_t* rank;
  double* dnext;
  double* dbest;
  double* hs;
  float* sb;
  float* sy;
  float* ppm;
  int16_t* mb;
  int16_t* my;
  int16_t* lb;
  int16_t* ly;
} vk_psm_out;

/* Optional per-candidate outputs, slot s*cap + j (j < n_cand[s], sorted by row); n_cand == NULL: not written;
 * hs == NULL: K2 outputs not written.  cap >= (pair_closure ? 2 : 1) * topk. */
typedef struct {
  int cap;
  int64_t* n_cand;
  int64_t* c_hyp;
  int64_t* c_row;
  int64_t* c_cnt;
  double* hs;
  float* sb;
  float* sy;
  float* ppm;
  int16_t* mb;
  int16_t* my;
  int16_t* lb;
  int16_t* ly;
} vk_cand_out;

/* Fused search of every work spectrum: K1 -> top-K + pair closure -> K2 -> ranking in one persistent kernel (one
 * CTA of `warps` warps per spectrum at a time, intermediate state in shared memory; `grid` CTAs, see
 * vk_search_fused_grid).  Same results as the staged entry points.  cnt_cap = window rows a spectrum may span in
 * total; spectra over it (or with more than 32 hypotheses) get status bit 1 and no PSMs -- search them with the
 * staged entry points.  status bit 2: a tile copy timed out.  work_counter (u32) and status (i32[n_spec]) are
 * zeroed by the call.  hyp_scored / hyp_matched may be NULL. */
int vk_search_fused(const vk_tindex* ix, const vk_frag_params* fp, const vk_fused_in* in, int warps, int cnt_cap,
                    int grid, unsigned int* work_counter, int32_t* status, int32_t* n_psm, int64_t* spec_scored,
                    int64_t* spec_matched, const vk_psm_out* psm, const vk_cand_out* cand, uint32_t* hyp_scored,
                    uint64_t* hyp_matched, void* stream);
/* Dynamic shared memory per CTA and the persistent grid size (CTAs resident per SM x SMs) of the fused search. */
int vk_search_fused_smem(const vk_tindex* ix, int warps, int topk, int pair_closure, int cnt_cap, int64_t* bytes);
int vk_search_fused_grid(const vk_tindex* ix, int warps, int topk, int pair_closure, int cnt_cap, int* grid);

/* ============================================================ Part 4: learned candidate pruner */

/* Features of n candidate hits (hypothesis, row, K1 count; e.g. the top-K shortlist of vk_select_topk with
 * pair_closure = 0, compacted): 16 BF16 per hit = the standardised (x - mu) / sd of K1 count, summed matched
 * intensity (isum of vk_k1_tiles / 2^24, a fraction of the TIC; isum[win_off[h] + row - lo[h]], or isum[i] for
 * candidate i when win_off is NULL, e.g. vk_select_hits' c_isum compacted), precursor error in ppm
 * ((M_hyp - mass32[row]) / mass32[row] * 1e6), charge, peptide length, missed cleavages; zero padded.
 * n bounds the buffers; when n_dev is given the device count *n_dev (<= n) is used instead (no host sync).  feat
 * 16-byte aligned (two 16-byte stores per hit). */
int vk_cand_features(int64_t n, const int64_t* n_dev, const int64_t* c_hyp, const int64_t* c_row,
                     const int64_t* c_cnt, const int64_t* win_off, const int64_t* h_lo, const uint32_t* isum,
                     const float* h_M, const int8_t* h_z, const float* mass32, const uint8_t* len,
                     const uint8_t* missed, const float* mu, const float* sd, void* feat_bf16, void* stream);
/* vk_compact_hits with the features on the way: the compacted hits as vk_compact_hits writes them (s_isum / c_isum
 * required) and, for every hit, the 16 standardised BF16 features vk_cand_features gives it, into feat (device,
 * 16-byte aligned, 16 BF16 per hit at the hit's compacted position; h_M, h_z the hypotheses' columns, mass32 /
 * length / missed the index rows'). */
int vk_compact_hits_features(int n_spec, int cap, const int64_t* n_cand, const int64_t* cand_off,
                             const int64_t* s_hyp, const int64_t* s_row, const int64_t* s_cnt, const uint32_t* s_isum,
                             const int8_t* h_maxfz, int64_t* c_hyp, int64_t* c_row, int64_t* c_cnt, int32_t* c_row32,
                             int8_t* c_maxfz, uint32_t* c_isum, const float* h_M, const int8_t* h_z,
                             const float* mass32, const uint8_t* len, const uint8_t* missed, const float* mu,
                             const float* sd, void* feat_bf16, void* stream);
/* MLP logits of n feature rows (16 BF16 each; n_dev as above): W1 [256 x 16] and W2 [256 x 256] BF16 row-major,
 * b1, b2, w3 (256) FP32, scalar b3; tensor cores (mma.sync BF16, FP32 accumulate); `grid` persistent CTAs of 256
 * threads, each holding the weights in vk_mlp_infer_smem() bytes of shared memory. */
int64_t vk_mlp_infer_smem(void);
int vk_mlp_infer(int64_t n, const int64_t* n_dev, const void* feat_bf16, const void* W1_bf16, const float* b1, const void* W2_bf16,
                 const float* b2, const float* w3, float b3, float* logit, int grid, void* stream);
/* The same logits on the 5th-generation tensor cores (tcgen05.mma, TMEM accumulators): tiles of 128 hits, layer 1
 * (K 16) and layer 2 (K 256) as UMMA from shared memory, bias / ReLU / BF16 rounding and the layer-3 dot in the
 * TMEM epilogues.  `grid` persistent CTAs of 512 threads (at most one per SM: vk_mlp_infer_tc_smem() bytes of
 * shared memory each).  `status` (device i32, zeroed by the caller) gets VK_STATUS_WAIT_TIMEOUT if an MMA did not
 * complete within the bounded wait. */
int64_t vk_mlp_infer_tc_smem(void);
int vk_mlp_infer_tc(int64_t n, const int64_t* n_dev, const void* feat_bf16, const void* W1_bf16, const float* b1,
                    const void* W2_bf16, const float* b2, const float* w3, float b3, float* logit, int grid,
                    int32_t* status, void* stream);
/* Pruned candidate selection per spectrum: hits with logit >= tau plus the min_keep best by (logit, count, hit
 * order) descending, at most max_keep (a power of two >= 16); pair closure; candidates sorted by row with duplicate
 * rows merged (lowest hypothesis, highest count) into slots s*cap (cap >= (pair_closure ? 2 : 1) * max_keep), the
 * layout of vk_select_topk.  max_hits (1..4096) bounds the hits of one spectrum (e.g. the shortlist's top-k); it
 * sizes the per-warp sort, and a spectrum with more hits keeps its first max_keep hits with logit >= tau in hit
 * order instead. */
int vk_select_pruned(int n_spec, const int64_t* spec_hyp_off, const int64_t* hit_off, const int64_t* hit_hyp,
                     const int32_t* hit_row, const int64_t* hit_cnt, const float* logit, float tau, int min_keep,
                     int max_keep, int pair_closure, const int64_t* partner, int cap, int max_hits, int64_t* c_hyp,
                     int64_t* c_row, int64_t* c_cnt, int64_t* n_cand, void* stream);

/* Training kernels.  vk_gemm: C[m*scm + n*scn] = sum_k A[m*sam + k*sak] * B[k*sbk + n*sbn] (+ bias[n]) (ReLU)
 * (rounded to a BF16 value); B is BF16 when b_bf16 != 0, else FP32; deterministic (fixed summation order). */
int vk_gemm(int M, int N, int K, const float* A, int64_t sam, int64_t sak, const void* B, int b_bf16, int64_t sbk,
            int64_t sbn, const float* bias, int relu, int round_bf16, float* C, int64_t scm, int64_t scn,
            void* stream);
/* The same product on the tcgen05 tensor cores: A and B rounded to BF16 as they are staged, FP32 accumulation in
 * TMEM (the tensor core's summation order, not vk_gemm's).  N a multiple of 16.  When the output tiles are few the K
 * range is split over CTAs: ws (device FP32, ws_floats >= vk_tc_gemm_ws_floats(M, N, K), may be NULL when that is
 * 0) takes the partial tiles, summed in split order by a second kernel.  status (device i32, not zeroed) gets
 * VK_STATUS_WAIT_TIMEOUT if an MMA did not complete within the bounded wait (the output is then not to be used). */
int64_t vk_tc_gemm_ws_floats(int M, int N, int K);
int vk_tc_gemm(int M, int N, int K, const float* A, int64_t sam, int64_t sak, const void* B, int b_bf16, int64_t sbk,
               int64_t sbn, const float* bias, int relu, int round_bf16, float* C, int64_t scm, int64_t scn,
               float* ws, int64_t ws_floats, int32_t* status, void* stream);
/* db[j] = sum_i dY[i, j], or sum_i v[i] dY[i, j] when v (device, n floats) is given: rows in chunks of 64 summed
 * sequentially, the chunk sums added in chunk order; ws (device, ws_floats >= vk_colsum_ws_floats(n, o)) holds the
 * chunk sums */
int64_t vk_colsum_ws_floats(int n, int o);
int vk_colsum(int n, int o, const float* dY, const float* v, float* ws, int64_t ws_floats, float* db, void* stream);
int vk_relu_mask(int64_t n, const float* Y, float* dY, void* stream);                  /* dY *= (Y > 0) */
/* weighted BCE with logits: dz = w (sigmoid(z) - y) inv_wsum; loss_part[ceil(n/256)] block partial sums */
int vk_bce(int n, const float* z, const float* y, const float* w, float inv_wsum, float* dz, float* loss_part,
           void* stream);
/* Adam step (step >= 1) on FP32 master weights, L2 term wd * p added to the gradient; writes the BF16 copy if
 * given */
int vk_adam(int64_t n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
            int step, float wd, void* p_bf16, void* stream);
int vk_to_bf16(int64_t n, const float* x, void* y, void* stream);
int vk_bf16_to_f32(int64_t n, const void* x, float* y, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* VULCAN_B200_H */
