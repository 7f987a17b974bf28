// See layout.hpp.
#include "layout.hpp"

#include <algorithm>
#include <numeric>
#include <stdexcept>
#include <thread>

namespace cuopt_b200 {

namespace {

// Internal order for `count` rows of the given lengths: long rows first (by length, descending,
// ties by original id), then the others sorted by length descending inside fixed windows.
std::vector<int> order_rows(const std::vector<int>& len, const layout_options& opt)
{
  const int count = (int)len.size();
  std::vector<int> lng, shrt;
  lng.reserve(64);
  shrt.reserve(count);
  for (int i = 0; i < count; ++i) (len[i] > opt.long_row_threshold ? lng : shrt).push_back(i);
  std::stable_sort(lng.begin(), lng.end(), [&](int a, int b) { return len[a] > len[b]; });
  const int w = std::max(32, opt.sort_window);
  for (size_t s = 0; s < shrt.size(); s += w) {
    auto first = shrt.begin() + s;
    auto last  = shrt.begin() + std::min(shrt.size(), s + (size_t)w);
    std::stable_sort(first, last, [&](int a, int b) { return len[a] > len[b]; });
  }
  std::vector<int> out;
  out.reserve(count);
  out.insert(out.end(), lng.begin(), lng.end());
  out.insert(out.end(), shrt.begin(), shrt.end());
  return out;
}

// Internal CSR (rows already in internal order) -> sliced ELL + long-row CSR.
void to_sell(int rows, int cols, int n_long, const std::vector<int64_t>& off,
             const std::vector<int>& idx, const std::vector<double>& val,
             const std::vector<int64_t>& src, sell_host& out)
{
  out.rows   = rows;
  out.cols   = cols;
  out.n_long = n_long;
  const int short_rows = rows - n_long;
  out.n_slices         = (short_rows + 31) / 32;
  out.long_off.resize(n_long + 1);
  for (int r = 0; r <= n_long; ++r) out.long_off[r] = off[r];
  const int64_t long_nnz = off[n_long];
  out.slice_off.resize(out.n_slices + 1);
  int64_t pos = long_nnz;
  for (int s = 0; s < out.n_slices; ++s) {
    out.slice_off[s] = pos;
    int mx           = 0;
    for (int t = 0; t < 32; ++t) {
      int r = n_long + s * 32 + t;
      if (r < rows) mx = std::max(mx, (int)(off[r + 1] - off[r]));
    }
    pos += (int64_t)mx * 32;
  }
  out.slice_off[out.n_slices] = pos;
  out.idx.assign(pos, 0);
  out.val.assign(pos, 0.0);
  out.src.assign(pos, -1);
  std::copy(idx.begin(), idx.begin() + long_nnz, out.idx.begin());
  std::copy(val.begin(), val.begin() + long_nnz, out.val.begin());
  std::copy(src.begin(), src.begin() + long_nnz, out.src.begin());

  auto fill = [&](int s0, int s1) {
    for (int s = s0; s < s1; ++s) {
      const int64_t base = out.slice_off[s];
      const int len      = (int)((out.slice_off[s + 1] - base) / 32);
      for (int t = 0; t < 32; ++t) {
        const int r = n_long + s * 32 + t;
        int64_t b = 0, e = 0;
        if (r < rows) {
          b = off[r];
          e = off[r + 1];
        }
        int last_idx = (e > b) ? idx[b] : 0;
        for (int k = 0; k < len; ++k) {
          const int64_t p = base + (int64_t)k * 32 + t;
          if (b + k < e) {
            out.idx[p] = idx[b + k];
            out.val[p] = val[b + k];
            out.src[p] = src[b + k];
            last_idx   = idx[b + k];
          } else {
            out.idx[p] = last_idx;  // padding re-reads a cached element, multiplies by 0
          }
        }
      }
    }
  };
  const int nthreads = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  if (out.n_slices < 4096 || nthreads == 1) {
    fill(0, out.n_slices);
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) {
      int s0 = (int)((int64_t)out.n_slices * t / nthreads);
      int s1 = (int)((int64_t)out.n_slices * (t + 1) / nthreads);
      pool.emplace_back(fill, s0, s1);
    }
    for (auto& th : pool) th.join();
  }
}

}  // namespace

lp_layout build_layout(int m, int n, const int* row_off, const int* col_idx, const double* val,
                       const layout_options& opt)
{
  lp_layout L;
  L.m   = m;
  L.n   = n;
  L.nnz = m > 0 ? (int64_t)row_off[m] : 0;

  std::vector<int> rlen(m), clen(n, 0);
  for (int i = 0; i < m; ++i) rlen[i] = row_off[i + 1] - row_off[i];
  for (int64_t k = 0; k < L.nnz; ++k) {
    const int j = col_idx[k];
    if (j < 0 || j >= n) throw std::invalid_argument("column index out of range");
    clen[j]++;
  }
  L.row_new2old = order_rows(rlen, opt);
  L.col_new2old = order_rows(clen, opt);
  L.row_old2new.resize(m);
  L.col_old2new.resize(n);
  for (int i = 0; i < m; ++i) L.row_old2new[L.row_new2old[i]] = i;
  for (int j = 0; j < n; ++j) L.col_old2new[L.col_new2old[j]] = j;

  // Internal CSR of A: rows in internal order, columns renamed, entries keep their order.
  std::vector<int64_t> aoff(m + 1, 0);
  for (int r = 0; r < m; ++r) aoff[r + 1] = aoff[r] + rlen[L.row_new2old[r]];
  std::vector<int> aidx(L.nnz);
  std::vector<double> aval(L.nnz);
  std::vector<int64_t> asrc(L.nnz);
  for (int r = 0; r < m; ++r) {
    const int o     = L.row_new2old[r];
    int64_t d       = aoff[r];
    for (int64_t k = row_off[o]; k < row_off[o + 1]; ++k, ++d) {
      aidx[d] = L.col_old2new[col_idx[k]];
      aval[d] = val[k];
      asrc[d] = k;
    }
  }
  // Internal CSR of A^T by counting sort over internal columns (entries ordered by internal row).
  std::vector<int64_t> toff(n + 1, 0);
  for (int c = 0; c < n; ++c) toff[c + 1] = toff[c] + clen[L.col_new2old[c]];
  std::vector<int> tidx(L.nnz);
  std::vector<double> tval(L.nnz);
  std::vector<int64_t> tsrc(L.nnz);
  {
    std::vector<int64_t> fillp(toff.begin(), toff.end() - 1);
    for (int r = 0; r < m; ++r)
      for (int64_t k = aoff[r]; k < aoff[r + 1]; ++k) {
        const int64_t d = fillp[aidx[k]]++;
        tidx[d]         = r;
        tval[d]         = aval[k];
        tsrc[d]         = asrc[k];
      }
  }
  int a_long = 0, t_long = 0;
  while (a_long < m && rlen[L.row_new2old[a_long]] > opt.long_row_threshold) ++a_long;
  while (t_long < n && clen[L.col_new2old[t_long]] > opt.long_row_threshold) ++t_long;
  to_sell(m, n, a_long, aoff, aidx, aval, asrc, L.a);
  to_sell(n, m, t_long, toff, tidx, tval, tsrc, L.at);
  return L;
}

}  // namespace cuopt_b200
