// Device CSR handle: upload, validation, symmetric expansion, row-block
// partition, lazy transpose and diagonal.
#include <algorithm>
#include <cstring>

#include "sb2_internal.cuh"
#include "sell.cuh"

namespace sb2 {

static int validate_csr(int m, int n, int nnz, const int* ptr, const int* ind,
                        int upper) {
  // Matrix_Sparse.cxx:118-170 (SELDON_CHECK_DIMENSIONS) plus the index checks
  // a device kernel needs to stay in bounds.
  if (ptr[0] != 0 || ptr[m] != nnz) return SB2_ERR_INVALID_CSR;
  for (int i = 0; i < m; i++) {
    if (ptr[i + 1] < ptr[i]) return SB2_ERR_INVALID_CSR;
    for (int k = ptr[i]; k < ptr[i + 1]; k++) {
      const int j = ind[k];
      if (j < 0 || j >= n) return SB2_ERR_INVALID_CSR;
      if (upper && j < i) return SB2_ERR_INVALID_CSR;
    }
  }
  return SB2_OK;
}

// Full operator from the stored upper triangle.  Row i lists first the
// mirrored strict-upper entries of rows k < i (increasing k), then row i's
// stored entries in stored order.
static void expand_symmetric(int m, const int* ptr, const int* ind,
                             const double* val, std::vector<int>& fptr,
                             std::vector<int>& find, std::vector<double>& fval) {
  std::vector<int> lower_cnt(m + 1, 0);
  for (int i = 0; i < m; i++)
    for (int k = ptr[i]; k < ptr[i + 1]; k++)
      if (ind[k] != i) lower_cnt[ind[k]]++;
  fptr.assign(m + 1, 0);
  for (int i = 0; i < m; i++) fptr[i + 1] = fptr[i] + lower_cnt[i] + (ptr[i + 1] - ptr[i]);
  const long long total = fptr[m];
  find.resize(total);
  fval.resize(total);
  std::vector<int> fill(m);
  for (int i = 0; i < m; i++) fill[i] = fptr[i];
  // mirrored entries, visited in increasing source row -> increasing k per row
  for (int i = 0; i < m; i++)
    for (int k = ptr[i]; k < ptr[i + 1]; k++) {
      const int j = ind[k];
      if (j != i) {
        find[fill[j]] = i;
        fval[fill[j]] = val[k];
        fill[j]++;
      }
    }
  for (int i = 0; i < m; i++)
    for (int k = ptr[i]; k < ptr[i + 1]; k++) {
      find[fill[i]] = ind[k];
      fval[fill[i]] = val[k];
      fill[i]++;
    }
}

int build_partition_host(const int* ptr, int rows, Partition* out) {
  std::vector<int> blk;
  std::vector<unsigned char> kind;
  blk.reserve(rows / 64 + 16);
  int r = 0;
  while (r < rows) {
    const int len0 = ptr[r + 1] - ptr[r];
    if (len0 > kLongRow) {
      blk.push_back(r);
      kind.push_back(kBlkLong);
      r++;
      continue;
    }
    const int start = r;
    int nnz = 0, maxlen = 0;
    while (r < rows && r - start < kRowCap) {
      const int len = ptr[r + 1] - ptr[r];
      if (len > kLongRow || nnz + len > kNnzCap) break;
      nnz += len;
      maxlen = std::max(maxlen, len);
      r++;
    }
    blk.push_back(start);
    kind.push_back(maxlen <= kThreadRowMax ? kBlkThread : kBlkWarp);
  }
  blk.push_back(rows);
  out->nblk = (int)kind.size();
  SB2_CUDA_TRY(cudaMalloc(&out->d_blk, sizeof(int) * blk.size()));
  SB2_CUDA_TRY(cudaMemcpy(out->d_blk, blk.data(), sizeof(int) * blk.size(), cudaMemcpyHostToDevice));
  if (out->nblk > 0) {
    SB2_CUDA_TRY(cudaMalloc(&out->d_kind, kind.size()));
    SB2_CUDA_TRY(cudaMemcpy(out->d_kind, kind.data(), kind.size(), cudaMemcpyHostToDevice));
  }
  return SB2_OK;
}

// Partition for the TMA-pipelined kernel: blocks of <= 2048 nonzeros and
// <= 512 rows; a row longer than 256 is a block of its own, summed by the
// whole CTA.  Not applicable (nblk = -1) when a row exceeds one stage.
int build_tma_partition_host(const int* ptr, int rows, Partition* out) {
  constexpr int kCap = 2048, kRowCapT = 512, kCtaRow = 256;
  std::vector<int> blk;
  std::vector<unsigned char> kind;
  int r = 0;
  while (r < rows) {
    const int len0 = ptr[r + 1] - ptr[r];
    if (len0 > kCap) {
      out->nblk = -1;
      return SB2_OK;
    }
    if (len0 > kCtaRow) {
      blk.push_back(r);
      kind.push_back(2);
      r++;
      continue;
    }
    const int start = r;
    int nnz = 0, maxlen = 0;
    while (r < rows && r - start < kRowCapT) {
      const int len = ptr[r + 1] - ptr[r];
      if (len > kCtaRow || nnz + len > kCap) break;
      nnz += len;
      maxlen = std::max(maxlen, len);
      r++;
    }
    blk.push_back(start);
    kind.push_back(maxlen <= kThreadRowMax ? 0 : 1);
  }
  blk.push_back(rows);
  out->nblk = (int)kind.size();
  SB2_CUDA_TRY(cudaMalloc(&out->d_blk, sizeof(int) * blk.size()));
  SB2_CUDA_TRY(cudaMemcpy(out->d_blk, blk.data(), sizeof(int) * blk.size(), cudaMemcpyHostToDevice));
  if (out->nblk > 0) {
    SB2_CUDA_TRY(cudaMalloc(&out->d_kind, kind.size()));
    SB2_CUDA_TRY(cudaMemcpy(out->d_kind, kind.data(), kind.size(), cudaMemcpyHostToDevice));
    std::vector<int4> desc(out->nblk);
    for (int b = 0; b < out->nblk; b++)
      desc[b] = make_int4(blk[b], blk[b + 1] | ((int)kind[b] << 30), ptr[blk[b]], ptr[blk[b + 1]]);
    SB2_CUDA_TRY(cudaMalloc(&out->d_desc, sizeof(int4) * desc.size()));
    SB2_CUDA_TRY(cudaMemcpy(out->d_desc, desc.data(), sizeof(int4) * desc.size(), cudaMemcpyHostToDevice));
  }
  return SB2_OK;
}

// Binned SELL-32: short rows in slices of 32 (sorted by length when the
// lengths are irregular), longer rows listed for the warp and CTA bins.
int build_sell_host(const int* ptr, const int* ind, const double* val, int rows,
                    SellArrays* out) {
  constexpr int kMax = 32, kCta = 1024, kRows = 128;
  std::vector<int> shortr, wr, cr;
  int lmin = kMax, lmax = 0;
  for (int i = 0; i < rows; i++) {
    const int len = ptr[i + 1] - ptr[i];
    if (len <= kMax) {
      shortr.push_back(i);
      lmin = std::min(lmin, len);
      lmax = std::max(lmax, len);
    } else if (len <= kCta) {
      wr.push_back(i);
    } else {
      cr.push_back(i);
    }
  }
  // sort only when the slices would otherwise carry much padding
  out->sorted = (lmax - lmin) > 8;
  if (out->sorted)
    std::stable_sort(shortr.begin(), shortr.end(), [&](int a, int b) {
      return (ptr[a + 1] - ptr[a]) > (ptr[b + 1] - ptr[b]);
    });
  const long long nshort = (long long)shortr.size();
  const int ns = (int)((nshort + kRows - 1) / kRows);
  auto row_at = [&](long long q) { return q < nshort ? shortr[q] : -1; };
  auto len_of = [&](int r) { return r < 0 ? 0 : ptr[r + 1] - ptr[r]; };
  // slice offsets in groups (a group = entry k of the 4 rows of one lane)
  std::vector<long long> sptr(ns + 1, 0);
  std::vector<uint2> qinfo((size_t)ns * 32);
  std::vector<int4> qrows((size_t)ns * 32);
  bool scattered = false;
  for (int sl = 0; sl < ns; sl++) {
    int w = 0;
    for (int l = 0; l < 32; l++) {
      const long long q0 = (long long)sl * kRows + 4 * l;
      int r[4];
      unsigned lens = 0;
      for (int j = 0; j < 4; j++) {
        r[j] = row_at(q0 + j);
        const int len = len_of(r[j]);
        w = std::max(w, len);
        lens |= (unsigned)len << (8 * j);
      }
      const bool consecutive = r[0] >= 0 && r[1] == r[0] + 1 && r[2] == r[0] + 2 && r[3] == r[0] + 3;
      uint2 inf;
      inf.x = consecutive ? (unsigned)r[0] : kQuadScattered;
      inf.y = lens;
      qinfo[(size_t)sl * 32 + l] = inf;
      qrows[(size_t)sl * 32 + l] = make_int4(r[0], r[1], r[2], r[3]);
      scattered = scattered || !consecutive;
    }
    sptr[sl + 1] = sptr[sl] + 32ll * w;
  }
  const long long tot = sptr[ns] * 4;  // entries incl. padding
  std::vector<int> scol(std::max(tot, 4ll), 0);
  std::vector<double> sval(std::max(tot, 4ll), 0.0);
  std::vector<long long> pos(std::max<long long>(ptr[rows], 1), -1);
  for (int sl = 0; sl < ns; sl++) {
    const int w = (int)((sptr[sl + 1] - sptr[sl]) / 32);
    for (int l = 0; l < 32; l++)
      for (int j = 0; j < 4; j++) {
        const int r = row_at((long long)sl * kRows + 4 * l + j);
        const int len = len_of(r);
        int last = 0;
        for (int k = 0; k < w; k++) {
          const long long e = (sptr[sl] + (long long)k * 32 + l) * 4 + j;
          if (k < len) {
            last = ind[ptr[r] + k];
            scol[e] = last;
            sval[e] = val[ptr[r] + k];
            pos[ptr[r] + k] = e;
          } else {
            scol[e] = last;  // padding: a column this row already reads, value 0, skipped
          }
        }
      }
  }
  out->nslice = ns;
  out->padded = tot;
  out->nwarp = (int)wr.size();
  out->ncta = (int)cr.size();
  SB2_CUDA_TRY(cudaMalloc(&out->d_sptr, sizeof(long long) * (ns + 1)));
  SB2_CUDA_TRY(cudaMemcpy(out->d_sptr, sptr.data(), sizeof(long long) * (ns + 1), cudaMemcpyHostToDevice));
  SB2_CUDA_TRY(cudaMalloc(&out->d_qinfo, sizeof(uint2) * std::max<size_t>(qinfo.size(), 1)));
  if (!qinfo.empty())
    SB2_CUDA_TRY(cudaMemcpy(out->d_qinfo, qinfo.data(), sizeof(uint2) * qinfo.size(), cudaMemcpyHostToDevice));
  if (scattered) {
    SB2_CUDA_TRY(cudaMalloc(&out->d_qrows, sizeof(int4) * qrows.size()));
    SB2_CUDA_TRY(cudaMemcpy(out->d_qrows, qrows.data(), sizeof(int4) * qrows.size(), cudaMemcpyHostToDevice));
  }
  SB2_CUDA_TRY(cudaMalloc(&out->d_scol, sizeof(int) * scol.size()));
  SB2_CUDA_TRY(cudaMemcpy(out->d_scol, scol.data(), sizeof(int) * scol.size(), cudaMemcpyHostToDevice));
  SB2_CUDA_TRY(cudaMalloc(&out->d_sval, sizeof(double) * sval.size()));
  SB2_CUDA_TRY(cudaMemcpy(out->d_sval, sval.data(), sizeof(double) * sval.size(), cudaMemcpyHostToDevice));
  SB2_CUDA_TRY(cudaMalloc(&out->d_pos, sizeof(long long) * pos.size()));
  SB2_CUDA_TRY(cudaMemcpy(out->d_pos, pos.data(), sizeof(long long) * pos.size(), cudaMemcpyHostToDevice));
  SB2_CUDA_TRY(cudaMalloc(&out->d_wrows, sizeof(int) * std::max<size_t>(wr.size(), 1)));
  if (!wr.empty()) SB2_CUDA_TRY(cudaMemcpy(out->d_wrows, wr.data(), sizeof(int) * wr.size(), cudaMemcpyHostToDevice));
  SB2_CUDA_TRY(cudaMalloc(&out->d_crows, sizeof(int) * std::max<size_t>(cr.size(), 1)));
  if (!cr.empty()) SB2_CUDA_TRY(cudaMemcpy(out->d_crows, cr.data(), sizeof(int) * cr.size(), cudaMemcpyHostToDevice));
  return SB2_OK;
}

void free_sell(SellArrays* s) {
  cudaFree(s->d_sptr);
  cudaFree(s->d_qinfo);
  cudaFree(s->d_qrows);
  cudaFree(s->d_scol);
  cudaFree(s->d_sval);
  cudaFree(s->d_sval32);
  cudaFree(s->d_wrows);
  cudaFree(s->d_crows);
  cudaFree(s->d_pos);
  *s = SellArrays();
}

int upload_csr(int rows, int cols, const int* ptr, const int* ind,
               const double* val, CsrArrays* out) {
  out->rows = rows;
  out->cols = cols;
  out->nnz = ptr[rows];
  const long long cap = padded_nnz(out->nnz);
  const long long pcap = padded_rows(rows);
  for (int i = 0; i < rows; i++) out->max_row = std::max(out->max_row, ptr[i + 1] - ptr[i]);
  SB2_CUDA_TRY(cudaMalloc(&out->d_ptr, sizeof(int) * pcap));
  SB2_CUDA_TRY(cudaMemset(out->d_ptr, 0, sizeof(int) * pcap));
  SB2_CUDA_TRY(cudaMalloc(&out->d_ind, sizeof(int) * cap));
  SB2_CUDA_TRY(cudaMalloc(&out->d_val, sizeof(double) * cap));
  SB2_CUDA_TRY(cudaMemcpy(out->d_ptr, ptr, sizeof(int) * (rows + 1), cudaMemcpyHostToDevice));
  // padding: column 0 with value 0 keeps every speculative vector load valid
  SB2_CUDA_TRY(cudaMemset(out->d_ind, 0, sizeof(int) * cap));
  SB2_CUDA_TRY(cudaMemset(out->d_val, 0, sizeof(double) * cap));
  if (out->nnz > 0) {
    SB2_CUDA_TRY(cudaMemcpy(out->d_ind, ind, sizeof(int) * out->nnz, cudaMemcpyHostToDevice));
    SB2_CUDA_TRY(cudaMemcpy(out->d_val, val, sizeof(double) * out->nnz, cudaMemcpyHostToDevice));
  }
  SB2_TRY(build_partition_host(ptr, rows, &out->part));
  SB2_TRY(build_sell_host(ptr, ind, val, rows, &out->sell));
  return build_tma_partition_host(ptr, rows, &out->tma);
}

void free_csr(CsrArrays* a) {
  cudaFree(a->d_ptr);
  cudaFree(a->d_ind);
  cudaFree(a->d_val);
  cudaFree(a->part.d_blk);
  cudaFree(a->part.d_kind);
  cudaFree(a->tma.d_blk);
  cudaFree(a->tma.d_kind);
  cudaFree(a->tma.d_desc);
  free_sell(&a->sell);
  *a = CsrArrays();
}

// A^T as a CSR (= CSC of A), entries of each column in increasing row order.
int ensure_transpose(const sb2_csr* cA) {
  sb2_csr* A = const_cast<sb2_csr*>(cA);
  std::lock_guard<std::mutex> g(A->mu);
  if (A->trans.d_ptr) return SB2_OK;
  const CsrArrays& f = A->full;
  std::vector<int> ptr(f.rows + 1), ind(f.nnz);
  std::vector<double> val(f.nnz);
  SB2_CUDA_TRY(cudaMemcpy(ptr.data(), f.d_ptr, sizeof(int) * (f.rows + 1), cudaMemcpyDeviceToHost));
  if (f.nnz) {
    SB2_CUDA_TRY(cudaMemcpy(ind.data(), f.d_ind, sizeof(int) * f.nnz, cudaMemcpyDeviceToHost));
    SB2_CUDA_TRY(cudaMemcpy(val.data(), f.d_val, sizeof(double) * f.nnz, cudaMemcpyDeviceToHost));
  }
  std::vector<int> tptr(f.cols + 1, 0), tind(f.nnz);
  std::vector<double> tval(f.nnz);
  for (long long k = 0; k < f.nnz; k++) tptr[ind[k] + 1]++;
  for (int c = 0; c < f.cols; c++) tptr[c + 1] += tptr[c];
  std::vector<int> fill(tptr.begin(), tptr.end() - 1);
  for (int i = 0; i < f.rows; i++)
    for (int k = ptr[i]; k < ptr[i + 1]; k++) {
      const int p = fill[ind[k]]++;
      tind[p] = i;
      tval[p] = val[k];
    }
  return upload_csr(f.cols, f.rows, tptr.data(), tind.data(), tval.data(), &A->trans);
}

__global__ void diag_kernel(int m, const int* __restrict__ ptr,
                            const int* __restrict__ ind,
                            const double* __restrict__ val, double* d) {
  // Matrix_Sparse::operator()(i, i) (Matrix_Sparse.cxx:1051-1083): advance
  // while k < b-1 and ind[k] < i, then test ind[k] == i.
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  int a = ptr[i], b = ptr[i + 1];
  double v = 0.0;
  if (a != b) {
    int k = a;
    while (k < b - 1 && ind[k] < i) k++;
    if (ind[k] == i) v = val[k];
  }
  d[i] = v;
}

int ensure_diag(const sb2_csr* cA) {
  sb2_csr* A = const_cast<sb2_csr*>(cA);
  std::lock_guard<std::mutex> g(A->mu);
  if (A->d_diag) return SB2_OK;
  double* d = nullptr;
  SB2_CUDA_TRY(cudaMalloc(&d, sizeof(double) * std::max(A->m, 1)));
  // The symmetric lookup scans the stored (upper) row, whose first entry is
  // the diagonal when present; the general lookup scans the full row.
  const CsrArrays& src = A->sym ? A->upper : A->full;
  if (A->m > 0)
    diag_kernel<<<(A->m + 255) / 256, 256>>>(A->m, src.d_ptr, src.d_ind, src.d_val, d);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    cudaFree(d);
    return map_cuda_error(e);
  }
  A->d_diag = d;
  return SB2_OK;
}

}  // namespace sb2

using namespace sb2;

extern "C" {

int sb2_csr_create(int m, int n, int nnz, const int* ptr, const int* ind,
                   const double* val, int symmetric_upper, int validate,
                   sb2_csr** out) try {
  SB2_TRACE("sb2_csr_create");
  if (!out || m < 0 || n < 0 || nnz < 0 || !ptr) return SB2_ERR_INVALID_VALUE;
  if (nnz > 0 && (!ind || !val)) return SB2_ERR_INVALID_VALUE;
  if (symmetric_upper && m != n) return SB2_ERR_INVALID_VALUE;
  *out = nullptr;
  // Device arrays (sb2_coo_to_csr's output, say) are read back first: the
  // validator and the slice layout are built on the host.
  cudaPointerAttributes pa;
  if (cudaPointerGetAttributes(&pa, ptr) == cudaSuccess && pa.type == cudaMemoryTypeDevice) {
    std::vector<int> hp(m + 1), hi(nnz);
    std::vector<double> hv(nnz);
    SB2_CUDA_TRY(cudaMemcpy(hp.data(), ptr, sizeof(int) * (m + 1), cudaMemcpyDeviceToHost));
    if (nnz > 0) {
      SB2_CUDA_TRY(cudaMemcpy(hi.data(), ind, sizeof(int) * nnz, cudaMemcpyDeviceToHost));
      SB2_CUDA_TRY(cudaMemcpy(hv.data(), val, sizeof(double) * nnz, cudaMemcpyDeviceToHost));
    }
    return sb2_csr_create(m, n, nnz, hp.data(), hi.data(), hv.data(), symmetric_upper, validate,
                          out);
  }
  cudaGetLastError();  // a host pointer unknown to CUDA is not an error
  if (validate) SB2_TRY(validate_csr(m, n, nnz, ptr, ind, symmetric_upper));
  else if (ptr[m] != nnz) return SB2_ERR_INVALID_CSR;

  std::unique_ptr<sb2_csr, int (*)(sb2_csr*)> A(new sb2_csr(), sb2_csr_destroy);
  A->device = current_device();
  A->m = m;
  A->n = n;
  A->nnz_stored = nnz;
  A->sym = symmetric_upper ? 1 : 0;
  int st;
  if (A->sym) {
    std::vector<int> fptr, find;
    std::vector<double> fval;
    expand_symmetric(m, ptr, ind, val, fptr, find, fval);
    st = upload_csr(m, n, fptr.data(), find.data(), fval.data(), &A->full);
    if (st == SB2_OK) st = upload_csr(m, n, ptr, ind, val, &A->upper);
  } else {
    st = upload_csr(m, n, ptr, ind, val, &A->full);
  }
  if (st != SB2_OK) return st;
  A->nnz = A->full.nnz;
  *out = A.release();
  return SB2_OK;
} SB2_CATCH

int sb2_csr_destroy(sb2_csr* A) try {
  if (!A) return SB2_OK;
  int prev = current_device();
  cudaSetDevice(A->device);
  free_csr(&A->full);
  free_csr(&A->upper);
  free_csr(&A->trans);
  cudaFree(A->d_diag);
  cudaFree(A->d_val32);
  cudaFree(A->d_diag32);
  cudaFree(A->d_hx);
  cudaFree(A->d_hy);
  for (int i = 0; i < 2; i++) {
    cudaFree(A->d_bx[i]);
    cudaFree(A->d_by[i]);
    if (A->e_in[i]) cudaEventDestroy(A->e_in[i]);
    if (A->e_kern[i]) cudaEventDestroy(A->e_kern[i]);
    if (A->e_out[i]) cudaEventDestroy(A->e_out[i]);
  }
  if (A->s_in) cudaStreamDestroy(A->s_in);
  if (A->s_out) cudaStreamDestroy(A->s_out);
  cudaSetDevice(prev);
  delete A;
  return SB2_OK;
} SB2_CATCH

int sb2_csr_info(const sb2_csr* A, int* m, int* n, int* nnz_stored, int* nnz_full) try {
  if (!A) return SB2_ERR_INVALID_VALUE;
  if (m) *m = A->m;
  if (n) *n = A->n;
  if (nnz_stored) *nnz_stored = A->nnz_stored;
  if (nnz_full) *nnz_full = (int)A->nnz;
  return SB2_OK;
} SB2_CATCH

int sb2_csr_download(const sb2_csr* A, int* ptr, int* ind, double* val) try {
  if (!A) return SB2_ERR_INVALID_VALUE;
  const CsrArrays& s = A->sym ? A->upper : A->full;
  if (ptr) SB2_CUDA_TRY(cudaMemcpy(ptr, s.d_ptr, sizeof(int) * (A->m + 1), cudaMemcpyDeviceToHost));
  if (ind && s.nnz) SB2_CUDA_TRY(cudaMemcpy(ind, s.d_ind, sizeof(int) * s.nnz, cudaMemcpyDeviceToHost));
  if (val && s.nnz) SB2_CUDA_TRY(cudaMemcpy(val, s.d_val, sizeof(double) * s.nnz, cudaMemcpyDeviceToHost));
  return SB2_OK;
} SB2_CATCH

}  // extern "C"
