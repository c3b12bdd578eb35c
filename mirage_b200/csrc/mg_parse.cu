// FASTA parse on the device: the query (or reference) file as the reference's loader reads it
// (Sequences::GetNumberOfHeaders / TReadFastaSequencesFromMem / SequenceToUpperCase,
// Sequences.cpp:283-320, 57-214, 43-55), as one pass over the whole file:
//   - the file must start with '>' (the reference stops with "0 Headers found" otherwise);
//   - each line starting with '>' is a header and starts a sequence;
//   - other lines are appended to the current sequence without a trailing '\r'; empty lines add
//     nothing; an unterminated last line counts like the others;
//   - a line starting with '@' is refused (the reference cannot load FASTQ: its loader counts
//     '>' headers only);
//   - sequence bytes are uppercased on request (bytes above 96, as signed char, lose 32).
// The reference splits large files into threads at header positions; in a file of more than
// 200 headers that makes consecutive headers without sequence lines share one sequence,
// depending on where the split falls. Here every header has its own sequence, as the reference
// gives for smaller files.
//
// Kernels: newline positions (select), one thread per line to classify it, scans for each
// line's sequence and output offset, one warp per data line to copy its bytes.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <cstdlib>
#include <string>

#include "mg_internal.h"

namespace mg {
namespace {

enum : int { kParseNoHeader = 1, kParseAt = 2, kParseLong = 4 };

// Newline flags, and their count (one atomic per block).
__global__ void __launch_bounds__(256) k_parse_flags(const uint8_t* text, uint64_t len, uint8_t* flag,
                                                     unsigned long long* count) {
  __shared__ unsigned long long s_n;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long n = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += stride) {
    const bool nl = text[i] == '\n';
    flag[i] = nl;
    n += nl;
  }
  atomicAdd(&s_n, n);
  __syncthreads();
  if (threadIdx.x == 0 && s_n) atomicAdd(count, s_n);
}

// Per line: raw start, data length (without '\r'), header flag, data byte count.
__global__ void k_parse_lines(const uint8_t* text, uint64_t len, const uint64_t* nl, uint64_t n_lines,
                              uint64_t* start, uint32_t* dlen, uint32_t* is_hdr, uint64_t* dbytes, int* err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_lines; j += stride) {
    const uint64_t s = j == 0 ? 0 : nl[j - 1] + 1;
    const uint64_t e = nl[j];  // one past the line (its '\n', or the end of the text)
    uint64_t n = e - s;
    if (n && text[e - 1] == '\r') n--;
    if (n > 0xFFFFFFFFull) {
      atomicOr(err, kParseLong);
      n = 0;
    }
    const bool raw_nonempty = e > s;
    const uint8_t c0 = raw_nonempty ? text[s] : 0;
    const bool hdr = c0 == '>';
    if (c0 == '@') atomicOr(err, kParseAt);
    if (j == 0 && !hdr) atomicOr(err, kParseNoHeader);
    start[j] = s;
    dlen[j] = (uint32_t)n;
    is_hdr[j] = hdr ? 1u : 0u;
    dbytes[j] = hdr ? 0ull : n;
  }
}

// Per header line: its sequence's first output byte and its text span.
__global__ void k_parse_heads(const uint64_t* start, const uint32_t* dlen, const uint32_t* is_hdr, const uint32_t* sid,
                              const uint64_t* ooff, uint64_t n_lines, uint64_t* seq_off, uint64_t* h_at, uint32_t* h_len) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_lines; j += stride)
    if (is_hdr[j]) {
      const uint32_t s = sid[j] - 1;
      seq_off[s] = ooff[j];
      h_at[s] = start[j];
      h_len[s] = dlen[j];
    }
}

// One warp per data line: its bytes to the output, uppercased on request.
__global__ void k_parse_copy(const uint8_t* text, const uint64_t* start, const uint32_t* dlen, const uint32_t* is_hdr,
                             const uint64_t* ooff, uint64_t n_lines, int upper, uint8_t* out) {
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  for (uint64_t j = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < n_lines; j += warps) {
    if (is_hdr[j]) continue;
    const uint8_t* src = text + start[j];
    uint8_t* dst = out + ooff[j];
    for (uint32_t t = lane; t < dlen[j]; t += 32) {
      uint8_t c = src[t];
      if (upper && (int8_t)c > 96) c = (uint8_t)(c - 32);
      dst[t] = c;
    }
  }
}

}  // namespace
}  // namespace mg

using namespace mg;

#define PCU(x)                                                                                       \
  do {                                                                                               \
    cudaError_t e_ = (x);                                                                            \
    if (e_ != cudaSuccess) return set_error(MG_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
  } while (0)

extern "C" void mg_seqs_free(mg_seqs* s) {
  if (!s) return;
  std::free(s->offsets);
  std::free(s->bases);
  std::free(s->header_at);
  std::free(s->header_len);
  *s = mg_seqs{};
}

extern "C" int mg_parse_fasta_device(int device, const uint8_t* text, uint64_t len, int uppercase, mg_seqs* out) {
  if (!out || (len && !text)) return set_error(MG_ERR_INVAL, "null argument");
  *out = mg_seqs{};
  auto fail_oom = [&]() {
    mg_seqs_free(out);
    return set_error(MG_ERR_OOM, "host memory for the parsed sequences");
  };
  out->offsets = (uint64_t*)std::calloc(1, 8);
  if (!out->offsets) return fail_oom();
  if (len == 0) return MG_OK;
  PCU(cudaSetDevice(device));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const unsigned grid = (unsigned)sms * 8;
  cudaStream_t st = 0;
  DevBuf d_text, d_flag, d_nl, d_nsel, tmp;
  if (d_text.alloc(len + 16) || d_flag.alloc(len + 16) || d_nsel.alloc(16)) return set_error(MG_ERR_OOM, "device memory for the parse");
  PCU(cudaMemcpy(d_text.p, text, len, cudaMemcpyHostToDevice));
  PCU(cudaMemset(d_nsel.p, 0, 16));
  k_parse_flags<<<grid, 256, 0, st>>>(d_text.as<uint8_t>(), len, d_flag.as<uint8_t>(),
                                       d_nsel.as<unsigned long long>() + 1);
  PCU(cudaGetLastError());
  // newline positions; the line count is theirs, plus an unterminated last line
  uint64_t n_nl = 0;
  {
    PCU(cudaMemcpy(&n_nl, d_nsel.as<unsigned long long>() + 1, 8, cudaMemcpyDeviceToHost));
    thrust::counting_iterator<uint64_t> idx(0);
    size_t tb_sel = 0;
    PCU(cub::DeviceSelect::Flagged(nullptr, tb_sel, idx, d_flag.as<uint8_t>(), (uint64_t*)nullptr,
                                   d_nsel.as<unsigned long long>(), (int64_t)len, st));
    if (tmp.alloc(tb_sel + 16) || d_nl.alloc((n_nl + 2) * 8))
      return set_error(MG_ERR_OOM, "device memory for the parse");
    PCU(cub::DeviceSelect::Flagged(tmp.p, tb_sel, idx, d_flag.as<uint8_t>(), d_nl.as<uint64_t>(),
                                   d_nsel.as<unsigned long long>(), (int64_t)len, st));
  }
  const bool tail = text[len - 1] != '\n';
  const uint64_t n_lines = n_nl + (tail ? 1 : 0);
  if (tail) PCU(cudaMemcpy(d_nl.as<uint64_t>() + n_nl, &len, 8, cudaMemcpyHostToDevice));
  if (n_lines >= 0xFFFFFFFFull) return set_error(MG_ERR_LIMIT, "more than 2^32-1 lines");
  d_flag.release();
  tmp.release();
  DevBuf d_start, d_dlen, d_hdr, d_dbytes, d_sid, d_ooff, d_err;
  if (d_start.alloc(n_lines * 8 + 8) || d_dlen.alloc(n_lines * 4 + 4) || d_hdr.alloc(n_lines * 4 + 4) ||
      d_dbytes.alloc(n_lines * 8 + 8) || d_sid.alloc(n_lines * 4 + 4) || d_ooff.alloc(n_lines * 8 + 8) ||
      d_err.alloc(4))
    return set_error(MG_ERR_OOM, "device memory for the parse");
  PCU(cudaMemset(d_err.p, 0, 4));
  k_parse_lines<<<grid, 256, 0, st>>>(d_text.as<uint8_t>(), len, d_nl.as<uint64_t>(), n_lines, d_start.as<uint64_t>(),
                                       d_dlen.as<uint32_t>(), d_hdr.as<uint32_t>(), d_dbytes.as<uint64_t>(),
                                       d_err.as<int>());
  PCU(cudaGetLastError());
  int err = 0;
  PCU(cudaMemcpy(&err, d_err.p, 4, cudaMemcpyDeviceToHost));
  if (err & kParseNoHeader) return set_error(MG_ERR_BADINPUT, "the file does not start with a FASTA header ('>')");
  if (err & kParseAt) return set_error(MG_ERR_BADINPUT, "a line starts with '@' (FASTQ is not read, as by the reference)");
  if (err & kParseLong) return set_error(MG_ERR_LIMIT, "a line longer than 2^32-1 bytes");
  {
    size_t t1 = 0, t2 = 0;
    PCU(cub::DeviceScan::InclusiveSum(nullptr, t1, d_hdr.as<uint32_t>(), d_sid.as<uint32_t>(), (int64_t)n_lines, st));
    PCU(cub::DeviceScan::ExclusiveSum(nullptr, t2, d_dbytes.as<uint64_t>(), d_ooff.as<uint64_t>(), (int64_t)n_lines, st));
    if (tmp.alloc((t1 > t2 ? t1 : t2) + 16)) return set_error(MG_ERR_OOM, "device memory for the parse");
    PCU(cub::DeviceScan::InclusiveSum(tmp.p, t1, d_hdr.as<uint32_t>(), d_sid.as<uint32_t>(), (int64_t)n_lines, st));
    PCU(cub::DeviceScan::ExclusiveSum(tmp.p, t2, d_dbytes.as<uint64_t>(), d_ooff.as<uint64_t>(), (int64_t)n_lines, st));
  }
  uint32_t n_seqs = 0;
  uint64_t last_off = 0, last_bytes = 0;
  PCU(cudaMemcpy(&n_seqs, d_sid.as<uint32_t>() + n_lines - 1, 4, cudaMemcpyDeviceToHost));
  PCU(cudaMemcpy(&last_off, d_ooff.as<uint64_t>() + n_lines - 1, 8, cudaMemcpyDeviceToHost));
  PCU(cudaMemcpy(&last_bytes, d_dbytes.as<uint64_t>() + n_lines - 1, 8, cudaMemcpyDeviceToHost));
  const uint64_t total = last_off + last_bytes;
  DevBuf d_soff, d_hat, d_hlen, d_out;
  if (d_soff.alloc(((uint64_t)n_seqs + 1) * 8) || d_hat.alloc((uint64_t)n_seqs * 8 + 8) ||
      d_hlen.alloc((uint64_t)n_seqs * 4 + 4) || d_out.alloc(total + 16))
    return set_error(MG_ERR_OOM, "device memory for the parse");
  k_parse_heads<<<grid, 256, 0, st>>>(d_start.as<uint64_t>(), d_dlen.as<uint32_t>(), d_hdr.as<uint32_t>(),
                                       d_sid.as<uint32_t>(), d_ooff.as<uint64_t>(), n_lines, d_soff.as<uint64_t>(),
                                       d_hat.as<uint64_t>(), d_hlen.as<uint32_t>());
  k_parse_copy<<<grid, 256, 0, st>>>(d_text.as<uint8_t>(), d_start.as<uint64_t>(), d_dlen.as<uint32_t>(),
                                      d_hdr.as<uint32_t>(), d_ooff.as<uint64_t>(), n_lines, uppercase, d_out.as<uint8_t>());
  PCU(cudaGetLastError());
  PCU(cudaMemcpy(d_soff.as<uint64_t>() + n_seqs, &total, 8, cudaMemcpyHostToDevice));
  std::free(out->offsets);
  out->offsets = (uint64_t*)std::malloc(((uint64_t)n_seqs + 1) * 8);
  out->bases = (uint8_t*)std::malloc(total ? total : 1);
  out->header_at = (uint64_t*)std::malloc((uint64_t)n_seqs * 8 + 8);
  out->header_len = (uint32_t*)std::malloc((uint64_t)n_seqs * 4 + 4);
  if (!out->offsets || !out->bases || !out->header_at || !out->header_len) return fail_oom();
  PCU(cudaMemcpy(out->offsets, d_soff.p, ((uint64_t)n_seqs + 1) * 8, cudaMemcpyDeviceToHost));
  if (total) PCU(cudaMemcpy(out->bases, d_out.p, total, cudaMemcpyDeviceToHost));
  if (n_seqs) {
    PCU(cudaMemcpy(out->header_at, d_hat.p, (uint64_t)n_seqs * 8, cudaMemcpyDeviceToHost));
    PCU(cudaMemcpy(out->header_len, d_hlen.p, (uint64_t)n_seqs * 4, cudaMemcpyDeviceToHost));
  }
  out->n_seqs = n_seqs;
  return MG_OK;
}
