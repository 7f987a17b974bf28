// See device_layout.cuh.
#include "device_layout.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <climits>
#include <stdexcept>

namespace cuopt_b200 {

namespace {

constexpr int kT = 256;

int grid_for(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>(1, (n + kT - 1) / kT), 1 << 20); }

__global__ void row_len_kernel(const int* off, int m, int* len)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    len[i] = off[i + 1] - off[i];
}

__global__ void col_count_kernel(const int* idx, int64_t nnz, int n, int* cnt, int* bad)
{
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int j = idx[k];
    if (j < 0 || j >= n)
      atomicExch(bad, 1);
    else
      atomicAdd(&cnt[j], 1);
  }
}

// Sort keys: long rows (len > thr) first by (instance, length descending); the rest by
// (instance, window, length descending).  `inst` (optional) gives each item's instance in a
// block-diagonal batch, so every instance's items stay contiguous inside each class; without it
// all items are instance 0.  A stable radix sort on these keys with values 0..count-1 keeps
// original order on ties, which makes the permutation deterministic.
__global__ void make_keys_kernel(const int* len, const int* inst, int count, int thr, int window,
                                 uint64_t* keys, int* ids, int* nlong)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const int l      = len[i];
    const uint64_t b = inst ? (uint64_t)inst[i] : 0ull;  // < 2^16
    uint64_t k;
    if (l > thr) {
      k = (b << 31) | (uint64_t)(INT_MAX - l);
      atomicAdd(nlong, 1);
    } else {
      k = (1ull << 63) | (b << 47) | ((uint64_t)(i / window) << 31) | (uint64_t)(thr - l);
    }
    keys[i] = k;
    ids[i]  = i;
  }
}

__global__ void invert_perm_kernel(const int* new2old, int count, int* old2new)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    old2new[new2old[i]] = i;
}

__global__ void gather_len_kernel(const int* len, const int* new2old, int count, int* out)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    out[i] = len[new2old[i]];
  if (blockIdx.x == 0 && threadIdx.x == 0) out[count] = 0;
}

// Internal CSR of A: warp per internal row.
__global__ void copy_rows_kernel(const int* uoff, const int* uidx, const double* uval,
                                 const int* row_new2old, const int* col_old2new, const int* noff,
                                 int m, int* aidx, double* aval, int* asrc, int* arow)
{
  const int lane = threadIdx.x & 31;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < m;
       r += (gridDim.x * blockDim.x) >> 5) {
    const int o = row_new2old[r];
    const int b = uoff[o], e = uoff[o + 1], d = noff[r];
    for (int k = lane; k < e - b; k += 32) {
      aidx[d + k] = col_old2new[uidx[b + k]];
      aval[d + k] = uval[b + k];
      asrc[d + k] = b + k;
      arow[d + k] = r;
    }
  }
}

__global__ void transpose_fill_kernel(const int* tpos, int64_t nnz, const int* arow,
                                      const double* aval, const int* asrc, int* tidx,
                                      double* tval, int* tsrc)
{
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nnz;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int k = tpos[p];
    tidx[p]     = arow[k];
    tval[p]     = aval[k];
    tsrc[p]     = asrc[k];
  }
}

// words[s] = 32 * (max row length in slice s); words[n_slices] = 0
__global__ void slice_words_kernel(const int* off, int rows, int n_long, int n_slices,
                                   int64_t* words)
{
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s <= n_slices; s += gridDim.x * blockDim.x) {
    if (s == n_slices) {
      words[s] = 0;
      continue;
    }
    int mx = 0;
    for (int t = 0; t < 32; ++t) {
      const int r = n_long + s * 32 + t;
      if (r < rows) mx = max(mx, off[r + 1] - off[r]);
    }
    words[s] = 32 * (int64_t)((mx + kChunk - 1) / kChunk * kChunk);
  }
}

__global__ void add_base_kernel(int64_t* v, int count, int64_t base)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    v[i] += base;
}

__global__ void long_off_kernel(const int* off, int n_long, int64_t* lo)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n_long; i += gridDim.x * blockDim.x)
    lo[i] = off[i];
}

// One warp per slice: lane t copies row (n_long + 32 s + t) into the column-major slots.
__global__ void sell_fill_kernel(const int* off, const int* idx, const double* val, const int* src,
                                 int rows, int n_long, int n_slices, const int64_t* slice_off,
                                 int* oidx, double* oval, int* osrc)
{
  const int lane = threadIdx.x & 31;
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < n_slices;
       s += (gridDim.x * blockDim.x) >> 5) {
    const int64_t base = slice_off[s];
    const int len      = (int)((slice_off[s + 1] - base) >> 5);
    const int r        = n_long + s * 32 + lane;
    int b = 0, e = 0;
    if (r < rows) {
      b = off[r];
      e = off[r + 1];
    }
    int last = (e > b) ? idx[b] : 0;
    for (int k = 0; k < len; ++k) {
      const int64_t p = sell_pos(base, k, lane);
      if (b + k < e) {
        last    = idx[b + k];
        oidx[p] = last;
        oval[p] = val[b + k];
        osrc[p] = src[b + k];
      } else {
        oidx[p] = last;
        oval[p] = 0.0;
        osrc[p] = -1;
      }
    }
  }
}

__global__ void iota_kernel(int* v, int64_t cnt)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt;
       i += (int64_t)gridDim.x * blockDim.x)
    v[i] = (int)i;
}

__global__ void gather_kernel(const double* src, const int* perm, int count, double sign,
                              double* dst)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    dst[i] = sign * src[perm[i]];
}
__global__ void scatter_kernel(const double* src, const int* perm, int count, double sign,
                               double* dst)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    dst[perm[i]] = sign * src[i];
}

struct temp_store {
  dbuf<char> buf;
  void* get(size_t bytes)
  {
    if (bytes > buf.size()) buf.resize(bytes);
    return buf.data();
  }
};

// Relabelling of `count` items with lengths `len` (device).  Returns the number of long items.
int order_items(const int* len, const int* inst, int count, const layout_params& p,
                cudaStream_t s, temp_store& tmp, dbuf<int>& new2old, dbuf<int>& old2new,
                int* d_counter, int* h_counter)
{
  dbuf<uint64_t> keys(count), keys_out(count);
  dbuf<int> ids(count);
  new2old.resize(count);
  old2new.resize(count);
  B200_CUDA_CHECK(cudaMemsetAsync(d_counter, 0, sizeof(int), s));
  make_keys_kernel<<<grid_for(count), kT, 0, s>>>(len, inst, count, p.long_threshold, p.window,
                                                  keys.data(), ids.data(), d_counter);
  B200_LAUNCH_CHECK();
  size_t bytes = 0;
  B200_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys.data(), keys_out.data(),
                                                  ids.data(), new2old.data(), count, 0, 64, s));
  B200_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(tmp.get(bytes), bytes, keys.data(),
                                                  keys_out.data(), ids.data(), new2old.data(),
                                                  count, 0, 64, s));
  invert_perm_kernel<<<grid_for(count), kT, 0, s>>>(new2old.data(), count, old2new.data());
  B200_CUDA_CHECK(cudaMemcpyAsync(h_counter, d_counter, sizeof(int), cudaMemcpyDeviceToHost, s));
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  return *h_counter;
}

// Internal CSR (offsets int32 rows+1, idx, val, src) -> dev_matrix
void to_sell(int rows, int cols, int n_long, const int* off, const int* idx, const double* val,
             const int* src, int64_t nnz, cudaStream_t s, temp_store& tmp, dev_matrix& M)
{
  M.rows     = rows;
  M.cols     = cols;
  M.n_long   = n_long;
  M.n_slices = (rows - n_long + 31) / 32;
  M.long_off.resize(n_long + 1);
  long_off_kernel<<<grid_for(n_long + 1), kT, 0, s>>>(off, n_long, M.long_off.data());
  int long_nnz = 0;
  B200_CUDA_CHECK(cudaMemcpyAsync(&long_nnz, off + n_long, sizeof(int), cudaMemcpyDeviceToHost, s));
  dbuf<int64_t> words(M.n_slices + 1);
  M.slice_off.resize(M.n_slices + 1);
  slice_words_kernel<<<grid_for(M.n_slices + 1), kT, 0, s>>>(off, rows, n_long, M.n_slices,
                                                             words.data());
  size_t bytes = 0;
  B200_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, words.data(), M.slice_off.data(),
                                                M.n_slices + 1, s));
  B200_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(tmp.get(bytes), bytes, words.data(),
                                                M.slice_off.data(), M.n_slices + 1, s));
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  // The sliced part starts on a 4-element boundary so its 128-bit loads are aligned.
  const int64_t sell_base = (long_nnz + kChunk - 1) / kChunk * kChunk;
  add_base_kernel<<<grid_for(M.n_slices + 1), kT, 0, s>>>(M.slice_off.data(), M.n_slices + 1,
                                                          sell_base);
  int64_t total = 0;
  B200_CUDA_CHECK(cudaMemcpyAsync(&total, M.slice_off.data() + M.n_slices, sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, s));
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  M.stored_count = total;
  M.idx.resize(std::max<int64_t>(total, 1));
  M.val.resize(std::max<int64_t>(total, 1));
  M.src.resize(std::max<int64_t>(total, 1));
  if (sell_base > long_nnz) {  // alignment gap: padding elements
    B200_CUDA_CHECK(cudaMemsetAsync(M.idx.data() + long_nnz, 0, (sell_base - long_nnz) * sizeof(int), s));
    B200_CUDA_CHECK(cudaMemsetAsync(M.val.data() + long_nnz, 0, (sell_base - long_nnz) * sizeof(double), s));
    B200_CUDA_CHECK(cudaMemsetAsync(M.src.data() + long_nnz, 0xFF, (sell_base - long_nnz) * sizeof(int), s));
  }
  if (long_nnz > 0) {
    B200_CUDA_CHECK(cudaMemcpyAsync(M.idx.data(), idx, long_nnz * sizeof(int), cudaMemcpyDeviceToDevice, s));
    B200_CUDA_CHECK(cudaMemcpyAsync(M.val.data(), val, long_nnz * sizeof(double), cudaMemcpyDeviceToDevice, s));
    B200_CUDA_CHECK(cudaMemcpyAsync(M.src.data(), src, long_nnz * sizeof(int), cudaMemcpyDeviceToDevice, s));
  }
  if (M.n_slices > 0)
    sell_fill_kernel<<<grid_for((int64_t)M.n_slices * 32), kT, 0, s>>>(
      off, idx, val, src, rows, n_long, M.n_slices, M.slice_off.data(), M.idx.data(),
      M.val.data(), M.src.data());
  B200_LAUNCH_CHECK();
  (void)nnz;
}

}  // namespace

void build_device_layout(int m, int n, const int* d_off, const int* d_idx, const double* d_val,
                         cudaStream_t s, device_layout& out, const layout_params& p)
{
  out.m = m;
  out.n = n;
  int nnz32 = 0;
  B200_CUDA_CHECK(cudaMemcpyAsync(&nnz32, d_off + m, sizeof(int), cudaMemcpyDeviceToHost, s));
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  const int64_t nnz = nnz32;
  out.nnz           = nnz;
  temp_store tmp;
  dbuf<int> counters(2);
  int* hcount = reinterpret_cast<int*>(pinned_scratch() + 32);

  dbuf<int> rlen(std::max(m, 1)), clen(std::max(n, 1));
  row_len_kernel<<<grid_for(m), kT, 0, s>>>(d_off, m, rlen.data());
  clen.zero(s);
  counters.zero(s);
  if (nnz > 0)
    col_count_kernel<<<grid_for(nnz), kT, 0, s>>>(d_idx, nnz, n, clen.data(), counters.data() + 1);
  B200_LAUNCH_CHECK();
  B200_CUDA_CHECK(cudaMemcpyAsync(hcount + 1, counters.data() + 1, sizeof(int),
                                  cudaMemcpyDeviceToHost, s));
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  if (hcount[1]) throw std::invalid_argument("constraint matrix column index out of range");
  trace_sync(s, "layout: lengths");

  const int a_long = order_items(rlen.data(), p.row_inst, m, p, s, tmp, out.row_new2old,
                                 out.row_old2new, counters.data(), hcount);
  const int t_long = order_items(clen.data(), p.col_inst, n, p, s, tmp, out.col_new2old,
                                 out.col_old2new, counters.data(), hcount);
  trace_sync(s, "layout: relabelling");

  // Internal A (CSR) ----------------------------------------------------------------------
  dbuf<int> alen(m + 1), aoff(m + 1);
  gather_len_kernel<<<grid_for(m + 1), kT, 0, s>>>(rlen.data(), out.row_new2old.data(), m,
                                                   alen.data());
  size_t bytes = 0;
  B200_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, alen.data(), aoff.data(), m + 1, s));
  B200_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(tmp.get(bytes), bytes, alen.data(), aoff.data(),
                                                m + 1, s));
  const int64_t nz = std::max<int64_t>(nnz, 1);
  dbuf<int> aidx(nz), asrc(nz), arow(nz);
  dbuf<double> aval(nz);
  copy_rows_kernel<<<grid_for((int64_t)m * 32), kT, 0, s>>>(
    d_off, d_idx, d_val, out.row_new2old.data(), out.col_old2new.data(), aoff.data(), m,
    aidx.data(), aval.data(), asrc.data(), arow.data());
  B200_LAUNCH_CHECK();

  trace_sync(s, "layout: internal A");
  // Internal A^T (CSR) by a stable sort of the entries on their internal column ----------------
  dbuf<int> tlen(n + 1), toff(n + 1), pos_in(nz), pos_out(nz), key_out(nz);
  gather_len_kernel<<<grid_for(n + 1), kT, 0, s>>>(clen.data(), out.col_new2old.data(), n,
                                                   tlen.data());
  B200_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, tlen.data(), toff.data(), n + 1, s));
  B200_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(tmp.get(bytes), bytes, tlen.data(), toff.data(),
                                                n + 1, s));
  dbuf<int> tidx(nz), tsrc(nz);
  dbuf<double> tval(nz);
  if (nnz > 0) {
    int bits = 1;
    while ((1ll << bits) < n) ++bits;
    iota_kernel<<<grid_for(nnz), kT, 0, s>>>(pos_in.data(), nnz);
    B200_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, aidx.data(), key_out.data(),
                                                    pos_in.data(), pos_out.data(), (int)nnz, 0,
                                                    bits, s));
    B200_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(tmp.get(bytes), bytes, aidx.data(),
                                                    key_out.data(), pos_in.data(), pos_out.data(),
                                                    (int)nnz, 0, bits, s));
    transpose_fill_kernel<<<grid_for(nnz), kT, 0, s>>>(pos_out.data(), nnz, arow.data(),
                                                       aval.data(), asrc.data(), tidx.data(),
                                                       tval.data(), tsrc.data());
    B200_LAUNCH_CHECK();
  }

  trace_sync(s, "layout: internal A^T");
  to_sell(m, n, a_long, aoff.data(), aidx.data(), aval.data(), asrc.data(), nnz, s, tmp, out.A);
  trace_sync(s, "layout: sliced A");
  to_sell(n, m, t_long, toff.data(), tidx.data(), tval.data(), tsrc.data(), nnz, s, tmp, out.AT);
  trace_sync(s, "layout: sliced A^T");
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
}

// One block per instance b of a batch whose arrays were uploaded instance by instance: row
// offsets and column indices become global (row_off[r0 + i + 1] += first non-zero of b;
// col_idx += first column of b) and every row / column records its instance.
__global__ void rebase_batch_kernel(const int* row_start, const int* col_start,
                                    const int* nnz_start, int* row_off, int* col_idx,
                                    int* row_inst, int* col_inst)
{
  const int b  = blockIdx.x;
  const int e0 = nnz_start[b], c0 = col_start[b];
  for (int i = row_start[b] + threadIdx.x; i < row_start[b + 1]; i += blockDim.x) {
    row_off[i + 1] += e0;
    row_inst[i] = b;
  }
  for (int j = c0 + threadIdx.x; j < col_start[b + 1]; j += blockDim.x) col_inst[j] = b;
  for (int k = e0 + threadIdx.x; k < nnz_start[b + 1]; k += blockDim.x) col_idx[k] += c0;
}

void rebase_batch_arrays(int count, const int* row_start, const int* col_start,
                         const int* nnz_start, int* row_off, int* col_idx, int* row_inst,
                         int* col_inst, cudaStream_t s)
{
  B200_CUDA_CHECK(cudaMemsetAsync(row_off, 0, sizeof(int), s));
  if (count > 0)
    rebase_batch_kernel<<<count, kT, 0, s>>>(row_start, col_start, nnz_start, row_off, col_idx,
                                             row_inst, col_inst);
  B200_LAUNCH_CHECK();
}

void permute_gather(const double* src, const int* perm, int count, double sign, double* dst,
                    cudaStream_t s)
{
  if (count > 0) gather_kernel<<<grid_for(count), kT, 0, s>>>(src, perm, count, sign, dst);
  B200_LAUNCH_CHECK();
}

void permute_scatter(const double* src, const int* perm, int count, double sign, double* dst,
                     cudaStream_t s)
{
  if (count > 0) scatter_kernel<<<grid_for(count), kT, 0, s>>>(src, perm, count, sign, dst);
  B200_LAUNCH_CHECK();
}

}  // namespace cuopt_b200
