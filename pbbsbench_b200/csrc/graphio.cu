// graphio.cu -- graph and sequence files.  The PBBS AdjacencyGraph text
// format (common/graphIO.h:191-215 reads it, :79-104 writes it) is tokenised
// and parsed on the device; integer sequences (the sequenceInt format of
// common/IO.h:198-203, the BFS driver's parent output) and graphs are
// formatted on the device; a binary CSR image loads and saves the arrays as
// they are.
//
// Text on the device: the bytes after the three header tokens are copied to
// HBM once.  A first pass counts token starts (a non-delimiter byte after a
// delimiter) per 4 KiB block, 16 bytes per thread; an exclusive scan of the
// block counts gives every block its first token index; a second pass finds
// the starts again, ranks them inside the block (block scan) and parses each
// token straight into the CSR arrays (token k < n: offsets[k], else
// edges[k - n]).  Both passes read the text once: bandwidth-bound.
#include <cuda_runtime.h>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cub/cub.cuh>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.cuh"

namespace pbg {
namespace {

constexpr int TX_THREADS = 256;
constexpr uint64_t TX_CHUNK = 16;                     // text bytes per thread
constexpr uint64_t TX_BLOCK = TX_THREADS * TX_CHUNK;  // 4 KiB of text per block
constexpr int FMT_PER_THREAD = 8;                     // values per thread when formatting
constexpr uint64_t FMT_BLOCK = (uint64_t)TX_THREADS * FMT_PER_THREAD;
constexpr uint64_t FMT_SLICE = 64ull << 20;           // values formatted per pass (bounds HBM use)
constexpr size_t STAGE_BYTES = 64ull << 20;           // pinned staging piece for file transfers
const char* ADJ_HEADER = "AdjacencyGraph";            // common/graphIO.h:73
const char* SEQ_INT_HEADER = "sequenceInt";           // common/IO.h:198

enum : unsigned { TXE_CHAR = 1u, TXE_RANGE = 2u, TXE_COUNT = 4u };

// The token delimiters of common/IO.h:41-50: space, tab, LF, CR and NUL.
__host__ __device__ __forceinline__ bool is_delim(uint32_t c) {
  return c == ' ' || c == '\n' || c == '\r' || c == '\t' || c == 0;
}

// Bit i set: byte c0 + i of the text starts a token.  Bytes past len read
// as NUL, a delimiter.
__device__ __forceinline__ uint32_t token_starts(const uint8_t* __restrict__ t, uint64_t len, uint64_t c0) {
  uint32_t w[4] = {0u, 0u, 0u, 0u};
  if (c0 + TX_CHUNK <= len) {
    const uint4 q = *reinterpret_cast<const uint4*>(t + c0);  // the buffer is 256-byte aligned
    w[0] = q.x;
    w[1] = q.y;
    w[2] = q.z;
    w[3] = q.w;
  } else {
    for (uint32_t i = 0; i < TX_CHUNK; i++)
      if (c0 + i < len) w[i / 4] |= (uint32_t)t[c0 + i] << (8 * (i % 4));
  }
  uint32_t d = 0;
#pragma unroll
  for (int i = 0; i < 16; i++) d |= (is_delim((w[i / 4] >> (8 * (i % 4))) & 0xFFu) ? 1u : 0u) << i;
  const uint32_t prev = (c0 == 0 || is_delim(t[c0 - 1])) ? 1u : 0u;
  return ~d & ((d << 1) | prev) & 0xFFFFu;
}

__global__ void k_count_tokens(const uint8_t* __restrict__ t, uint64_t len, unsigned long long* __restrict__ cnt) {
  using BR = cub::BlockReduce<uint32_t, TX_THREADS>;
  __shared__ typename BR::TempStorage tmp;
  const uint64_t c0 = ((uint64_t)blockIdx.x * TX_THREADS + threadIdx.x) * TX_CHUNK;
  const uint32_t c = (c0 < len) ? (uint32_t)__popc(token_starts(t, len, c0)) : 0u;
  const uint32_t s = BR(tmp).Sum(c);
  if (threadIdx.x == 0) cnt[blockIdx.x] = s;
}

// Parses every token of the block's text: decimal digits only (leading
// zeros allowed), value < 2^32.  Token k goes to off[k] (k < n) or
// edg[k - n] (k < n + m).
__global__ void k_parse_tokens(const uint8_t* __restrict__ t, uint64_t len,
                               const unsigned long long* __restrict__ base, uint32_t n, uint64_t m,
                               uint32_t* __restrict__ off, uint32_t* __restrict__ edg, unsigned* err) {
  using BS = cub::BlockScan<uint32_t, TX_THREADS>;
  __shared__ typename BS::TempStorage tmp;
  const uint64_t c0 = ((uint64_t)blockIdx.x * TX_THREADS + threadIdx.x) * TX_CHUNK;
  uint32_t st = (c0 < len) ? token_starts(t, len, c0) : 0u;
  uint32_t rank = 0;
  BS(tmp).ExclusiveSum((uint32_t)__popc(st), rank);
  uint64_t k = base[blockIdx.x] + rank;
  unsigned e = 0;
  while (st) {
    uint64_t p = c0 + (uint64_t)(__ffs(st) - 1);
    st &= st - 1;
    uint64_t v = 0;
    int nd = 0;
    bool bad = false;
    for (; p < len; p++) {
      const uint32_t c = t[p];
      if (is_delim(c)) break;
      if (c < '0' || c > '9') {
        bad = true;
        break;
      }
      if (nd > 0 || c != '0') nd++;
      if (nd > 10) {  // 11 significant digits: >= 10^10
        bad = true;
        break;
      }
      v = v * 10 + (c - '0');
    }
    if (bad)
      e |= (nd > 10) ? TXE_RANGE : TXE_CHAR;
    else if (v > 0xFFFFFFFFull)
      e |= TXE_RANGE;
    else if (k < n)
      off[k] = (uint32_t)v;
    else if (k - n < m)
      edg[k - n] = (uint32_t)v;
    else
      e |= TXE_COUNT;
    k++;
  }
  if (e) atomicOr(err, e);
}

__host__ __device__ __forceinline__ uint32_t ndigits(uint32_t x) {
  uint32_t d = 1;
  for (uint64_t p = 10; p <= x && d < 10; p *= 10) d++;
  return d;
}

// Characters of value i: its decimal digits, a '-' first for a negative
// signed value, and the '\n' that follows it.
template <bool SIGNED>
__device__ __forceinline__ uint32_t text_len(uint32_t x) {
  if (SIGNED && (int32_t)x < 0) return 2 + ndigits((uint32_t)(-(int64_t)(int32_t)x));
  return 1 + ndigits(x);
}

template <bool SIGNED>
__global__ void k_text_len(const uint32_t* __restrict__ v, uint64_t cnt, unsigned long long* __restrict__ blen) {
  using BR = cub::BlockReduce<unsigned long long, TX_THREADS>;
  __shared__ typename BR::TempStorage tmp;
  const uint64_t i0 = ((uint64_t)blockIdx.x * TX_THREADS + threadIdx.x) * FMT_PER_THREAD;
  unsigned long long s = 0;
  for (int j = 0; j < FMT_PER_THREAD; j++)
    if (i0 + j < cnt) s += text_len<SIGNED>(v[i0 + j]);
  s = BR(tmp).Sum(s);
  if (threadIdx.x == 0) blen[blockIdx.x] = s;
}

template <bool SIGNED>
__global__ void k_text_write(const uint32_t* __restrict__ v, uint64_t cnt, const unsigned long long* __restrict__ base,
                             char* __restrict__ out) {
  // the block's text is built in shared memory, then copied out with
  // consecutive threads on consecutive bytes (coalesced stores)
  constexpr int MAX_CHARS = TX_THREADS * FMT_PER_THREAD * 12;  // '-', 10 digits, '\n'
  using BS = cub::BlockScan<unsigned int, TX_THREADS>;
  __shared__ typename BS::TempStorage tmp;
  __shared__ char buf[MAX_CHARS];
  __shared__ unsigned int s_total;
  const uint64_t i0 = ((uint64_t)blockIdx.x * TX_THREADS + threadIdx.x) * FMT_PER_THREAD;
  unsigned int s = 0;
  for (int j = 0; j < FMT_PER_THREAD; j++)
    if (i0 + j < cnt) s += text_len<SIGNED>(v[i0 + j]);
  unsigned int pos = 0, total = 0;
  BS(tmp).ExclusiveSum(s, pos, total);
  if (threadIdx.x == 0) s_total = total;
  for (int j = 0; j < FMT_PER_THREAD; j++) {
    if (i0 + j >= cnt) break;
    uint32_t x = v[i0 + j];
    if (SIGNED && (int32_t)x < 0) {
      buf[pos++] = '-';
      x = (uint32_t)(-(int64_t)(int32_t)x);
    }
    const uint32_t d = ndigits(x);
    for (uint32_t q = d; q > 0; q--) {
      buf[pos + q - 1] = (char)('0' + x % 10);
      x /= 10;
    }
    pos += d;
    buf[pos++] = '\n';
  }
  __syncthreads();
  char* dst = out + base[blockIdx.x];
  for (unsigned int i = threadIdx.x; i < s_total; i += TX_THREADS) dst[i] = buf[i];
}

// The three header tokens of a text (header word, n, m) from its first
// `avail` bytes; `body` = the offset just past the third token.
int parse_header(const char* p, uint64_t avail, const char* want, uint64_t* vals, int nvals, uint64_t* body) {
  uint64_t i = 0;
  for (int tok = 0; tok <= nvals; tok++) {
    while (i < avail && is_delim((uint8_t)p[i])) i++;
    const uint64_t b = i;
    while (i < avail && !is_delim((uint8_t)p[i])) i++;
    if (i == b)
      return fail(PBG_ERR_ARG, tok == 0 ? std::string("bad input: no ") + want + " header"
                                        : std::string("bad input: the header has no value ") + std::to_string(tok));
    if (i == avail && avail >= STAGE_BYTES) return fail(PBG_ERR_ARG, "bad input: header token too long");
    if (tok == 0) {
      if (i - b != strlen(want) || memcmp(p + b, want, i - b) != 0)
        return fail(PBG_ERR_ARG, std::string("bad input: missing header ") + want);
      continue;
    }
    uint64_t v = 0;
    for (uint64_t j = b; j < i; j++) {
      const char c = p[j];
      if (c < '0' || c > '9' || v > (~0ull - 9) / 10)
        return fail(PBG_ERR_ARG, std::string("bad input: header value ") + std::to_string(tok) + " is not a count");
      v = v * 10 + (uint64_t)(c - '0');
    }
    vals[tok - 1] = v;
  }
  *body = i;
  return PBG_OK;
}

struct DevMem {
  void* p = nullptr;
  ~DevMem() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 1); }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Two pinned pieces and their copy events.  Pinning 128 MiB costs tens of
// milliseconds, so the pieces are kept for the process (one set per device)
// and a transfer holds them for its duration; a transfer that finds them in
// use pins its own.
struct StagePool {
  std::mutex mu;
  char* h[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool busy = false;
};
StagePool g_stage[16];

struct Stage {
  char* h[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  StagePool* pool = nullptr;  // the pieces are the pool's (returned, not freed)
  ~Stage() {
    for (int i = 0; i < 2; i++)
      if (ev[i]) cudaEventSynchronize(ev[i]);
    if (pool) {
      std::lock_guard<std::mutex> lk(pool->mu);
      pool->busy = false;
      return;
    }
    for (int i = 0; i < 2; i++) {
      if (ev[i]) cudaEventDestroy(ev[i]);
      if (h[i]) cudaFreeHost(h[i]);
    }
  }
  cudaError_t pin() {
    for (int i = 0; i < 2; i++) {
      cudaError_t e = cudaHostAlloc(&h[i], STAGE_BYTES, cudaHostAllocDefault);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  cudaError_t init() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 16) return pin();
    StagePool& P = g_stage[dev];
    {
      std::lock_guard<std::mutex> lk(P.mu);
      if (P.busy) return pin();
      if (!P.h[0]) {
        e = pin();
        if (e != cudaSuccess) return e;  // the partial pieces are freed by the destructor
        P.h[0] = h[0];
        P.h[1] = h[1];
        P.ev[0] = ev[0];
        P.ev[1] = ev[1];
      }
      P.busy = true;
    }
    pool = &P;
    for (int i = 0; i < 2; i++) {
      h[i] = P.h[i];
      ev[i] = P.ev[i];
    }
    return cudaSuccess;
  }
};

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

// CSR from the text body (the bytes after the header tokens) now on the device.
int parse_body(const uint8_t* d_text, uint64_t len, uint64_t n64, uint64_t m64, uint32_t flags, int num_sms,
               cudaStream_t s, pbg_graph** out) {
  if (n64 == 0 || n64 > PBG_MAX_VERTICES) return fail(PBG_ERR_ARG, "bad input: n must be in [1, 2^31)");
  if (m64 > 0xFFFFFFFFull) return fail(PBG_ERR_ARG, "bad input: m must fit in 32 bits");
  const uint32_t n = (uint32_t)n64;
  const uint64_t nblk = (len + TX_BLOCK - 1) / TX_BLOCK;
  DevMem cnt, base, err, tmp;
  unsigned long long total = 0;
  if (nblk) {
    PBG_CUDA(cnt.alloc(sizeof(unsigned long long) * nblk));
    PBG_CUDA(base.alloc(sizeof(unsigned long long) * nblk));
    k_count_tokens<<<(unsigned)nblk, TX_THREADS, 0, s>>>(d_text, len, cnt.as<unsigned long long>());
    PBG_CUDA(cudaGetLastError());
    size_t tb = 0;
    PBG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.as<unsigned long long>(), base.as<unsigned long long>(),
                                           (int64_t)nblk, s));
    PBG_CUDA(tmp.alloc(tb));
    PBG_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.as<unsigned long long>(), base.as<unsigned long long>(),
                                           (int64_t)nblk, s));
    unsigned long long last[2] = {0, 0};
    PBG_CUDA(cudaMemcpyAsync(&last[0], base.as<unsigned long long>() + nblk - 1, sizeof(last[0]),
                             cudaMemcpyDeviceToHost, s));
    PBG_CUDA(cudaMemcpyAsync(&last[1], cnt.as<unsigned long long>() + nblk - 1, sizeof(last[1]),
                             cudaMemcpyDeviceToHost, s));
    PBG_CUDA(cudaStreamSynchronize(s));
    total = last[0] + last[1];
  }
  // the reference's check (common/graphIO.h:203-205), counting the header's three tokens
  if (total != n64 + m64)
    return fail(PBG_ERR_ARG, "bad input file: length = " + std::to_string(total + 3) +
                                 " n+m+3 = " + std::to_string(n64 + m64 + 3));
  pbg_graph* g = nullptr;
  int rc = new_handle(n, m64, flags, &g);
  if (rc) return rc;
  unsigned h_err = 0;
  const uint32_t m32 = (uint32_t)m64;
  cudaError_t e = err.alloc(sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemsetAsync(err.p, 0, sizeof(unsigned), g->stream);
  // the handle's stream runs after the counting pass on s
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && nblk) {
    k_parse_tokens<<<(unsigned)nblk, TX_THREADS, 0, g->stream>>>(d_text, len, base.as<unsigned long long>(), n, m64,
                                                               g->d_offsets, g->d_edges, err.as<unsigned>());
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)  // offsets[n] = m: the tag of common/graphIO.h:207-209
    e = cudaMemcpyAsync(g->d_offsets + n, &m32, sizeof(uint32_t), cudaMemcpyHostToDevice, g->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, err.p, sizeof(unsigned), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) {
    pbg_graph_free(g);
    return cuda_fail(e, "graph text parse");
  }
  if (h_err) {
    pbg_graph_free(g);
    if (h_err & TXE_CHAR) return fail(PBG_ERR_ARG, "bad input: a token is not an unsigned decimal integer");
    if (h_err & TXE_RANGE) return fail(PBG_ERR_ARG, "bad input: a value does not fit in 32 bits");
    return fail(PBG_ERR_ARG, "bad input: token count");
  }
  rc = finish_graph(g);
  if (rc) {
    pbg_graph_free(g);
    return rc;
  }
  *out = g;
  return PBG_OK;
}

int device_of(int* num_sms) {
  int dev = 0;
  PBG_CUDA(cudaGetDevice(&dev));
  PBG_CUDA(cudaDeviceGetAttribute(num_sms, cudaDevAttrMultiProcessorCount, dev));
  return PBG_OK;
}

struct StreamHold {
  cudaStream_t s = nullptr;
  ~StreamHold() {
    if (s) cudaStreamDestroy(s);
  }
};

// Writes cnt device values as decimal text, one per line, to f: FMT_SLICE
// values at a time are formatted on the device and copied out through the
// pinned pieces.
int write_values(FILE* f, const uint32_t* d_vals, uint64_t cnt, bool is_signed, Stage& st, cudaStream_t s) {
  for (uint64_t v0 = 0; v0 < cnt; v0 += FMT_SLICE) {
    const uint64_t c = std::min<uint64_t>(FMT_SLICE, cnt - v0);
    const uint64_t nblk = (c + FMT_BLOCK - 1) / FMT_BLOCK;
    DevMem blen, base, tmp, text;
    PBG_CUDA(blen.alloc(sizeof(unsigned long long) * nblk));
    PBG_CUDA(base.alloc(sizeof(unsigned long long) * nblk));
    if (is_signed)
      k_text_len<true><<<(unsigned)nblk, TX_THREADS, 0, s>>>(d_vals + v0, c, blen.as<unsigned long long>());
    else
      k_text_len<false><<<(unsigned)nblk, TX_THREADS, 0, s>>>(d_vals + v0, c, blen.as<unsigned long long>());
    PBG_CUDA(cudaGetLastError());
    size_t tb = 0;
    PBG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, blen.as<unsigned long long>(), base.as<unsigned long long>(),
                                           (int64_t)nblk, s));
    PBG_CUDA(tmp.alloc(tb));
    PBG_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, blen.as<unsigned long long>(), base.as<unsigned long long>(),
                                           (int64_t)nblk, s));
    unsigned long long last[2] = {0, 0};
    PBG_CUDA(cudaMemcpyAsync(&last[0], base.as<unsigned long long>() + nblk - 1, sizeof(last[0]),
                             cudaMemcpyDeviceToHost, s));
    PBG_CUDA(cudaMemcpyAsync(&last[1], blen.as<unsigned long long>() + nblk - 1, sizeof(last[1]),
                             cudaMemcpyDeviceToHost, s));
    PBG_CUDA(cudaStreamSynchronize(s));
    const uint64_t bytes = last[0] + last[1];
    PBG_CUDA(text.alloc(bytes));
    if (is_signed)
      k_text_write<true><<<(unsigned)nblk, TX_THREADS, 0, s>>>(d_vals + v0, c, base.as<unsigned long long>(),
                                                               text.as<char>());
    else
      k_text_write<false><<<(unsigned)nblk, TX_THREADS, 0, s>>>(d_vals + v0, c, base.as<unsigned long long>(),
                                                                text.as<char>());
    PBG_CUDA(cudaGetLastError());
    // out through the two pinned pieces: copy piece i + 1 while piece i is written
    uint64_t done = 0;
    int cur = 0;
    uint64_t piece[2] = {0, 0};
    while (done < bytes || piece[cur ^ 1]) {
      if (done < bytes) {
        piece[cur] = std::min<uint64_t>(STAGE_BYTES, bytes - done);
        PBG_CUDA(cudaMemcpyAsync(st.h[cur], text.as<char>() + done, piece[cur], cudaMemcpyDeviceToHost, s));
        PBG_CUDA(cudaEventRecord(st.ev[cur], s));
        done += piece[cur];
      }
      const int prev = cur ^ 1;
      if (piece[prev]) {
        PBG_CUDA(cudaEventSynchronize(st.ev[prev]));
        if (fwrite(st.h[prev], 1, piece[prev], f) != piece[prev]) return fail(PBG_ERR_ARG, "file write failed");
        piece[prev] = 0;
      }
      cur ^= 1;
    }
  }
  return PBG_OK;
}

// Bytes to move into HBM: a file (read with pread) or host memory.
struct Source {
  int fd = -1;
  const char* mem = nullptr;
};

bool fill_part(const Source& src, char* dst, uint64_t off, uint64_t len) {
  if (src.mem) {
    memcpy(dst, src.mem + off, len);
    return true;
  }
  while (len) {
    const ssize_t r = pread(src.fd, dst, len, (off_t)off);
    if (r <= 0) return false;
    dst += r;
    off += (uint64_t)r;
    len -= (uint64_t)r;
  }
  return true;
}

// [off, off + len) of the source into dst, by up to 8 host threads (a page
// cache copy or a memcpy runs at a few GB/s per thread, below the PCIe link).
bool parallel_fill(const Source& src, char* dst, uint64_t off, uint64_t len) {
  constexpr uint64_t MIN_PART = 4ull << 20;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned nt = (unsigned)std::min<uint64_t>(std::min(8u, hw), (len + MIN_PART - 1) / MIN_PART);
  if (nt <= 1) return fill_part(src, dst, off, len);
  const uint64_t part = (len + nt - 1) / nt;
  std::atomic<bool> ok{true};
  std::vector<std::thread> th;
  for (unsigned k = 1; k < nt; k++) {
    const uint64_t a = k * part, b = std::min(len, a + part);
    if (a < b) th.emplace_back([&, a, b] {
        if (!fill_part(src, dst + a, off + a, b - a)) ok = false;
      });
  }
  if (!fill_part(src, dst, off, std::min(len, part))) ok = false;
  for (auto& t : th) t.join();
  return ok;
}

// Moves `bytes` from the source (at src_off) into device memory through the
// pinned pieces: the fill of piece i + 1 overlaps the copy of piece i.
int to_device(const Source& src, uint64_t src_off, uint64_t bytes, char* dst, Stage& st, cudaStream_t s) {
  uint64_t done = 0;
  int cur = 0;
  while (done < bytes) {
    const uint64_t c = std::min<uint64_t>(STAGE_BYTES, bytes - done);
    PBG_CUDA(cudaEventSynchronize(st.ev[cur]));  // the piece's previous copy is done
    if (!parallel_fill(src, st.h[cur], src_off + done, c))
      return fail(PBG_ERR_ARG, "file read failed (shorter than its header says?)");
    PBG_CUDA(cudaMemcpyAsync(dst + done, st.h[cur], c, cudaMemcpyHostToDevice, s));
    PBG_CUDA(cudaEventRecord(st.ev[cur], s));
    done += c;
    cur ^= 1;
  }
  PBG_CUDA(cudaStreamSynchronize(s));
  return PBG_OK;
}

struct Fd {
  int fd = -1;
  ~Fd() {
    if (fd >= 0) close(fd);
  }
};

int device_to_file(FILE* f, const char* src, uint64_t bytes, Stage& st, cudaStream_t s) {
  uint64_t done = 0;
  int cur = 0;
  uint64_t piece[2] = {0, 0};
  while (done < bytes || piece[cur ^ 1]) {
    if (done < bytes) {
      piece[cur] = std::min<uint64_t>(STAGE_BYTES, bytes - done);
      PBG_CUDA(cudaMemcpyAsync(st.h[cur], src + done, piece[cur], cudaMemcpyDeviceToHost, s));
      PBG_CUDA(cudaEventRecord(st.ev[cur], s));
      done += piece[cur];
    }
    const int prev = cur ^ 1;
    if (piece[prev]) {
      PBG_CUDA(cudaEventSynchronize(st.ev[prev]));
      if (fwrite(st.h[prev], 1, piece[prev], f) != piece[prev]) return fail(PBG_ERR_ARG, "file write failed");
      piece[prev] = 0;
    }
    cur ^= 1;
  }
  return PBG_OK;
}

// Binary CSR image: this header, then uint32 offsets[n + 1], uint32 edges[m]
// (little-endian, as in memory).
struct BinHeader {
  char magic[8];
  uint64_t n;
  uint64_t m;
  uint32_t flags;  // PBG_GRAPH_SYMMETRIC when the saved graph was symmetric
  uint32_t reserved;
};
const char BIN_MAGIC[8] = {'P', 'B', 'G', 'C', 'S', 'R', '0', '1'};

}  // namespace
}  // namespace pbg

using namespace pbg;

extern "C" int pbg_graph_parse_adj(const char* text, uint64_t len, uint32_t flags, pbg_graph** out) {
  if (!text || !out) return fail(PBG_ERR_ARG, "NULL argument");
  uint64_t nm[2] = {0, 0}, body = 0;
  int rc = parse_header(text, std::min<uint64_t>(len, STAGE_BYTES), ADJ_HEADER, nm, 2, &body);
  if (rc) return rc;
  if (nm[0] == 0 || nm[0] > PBG_MAX_VERTICES) return fail(PBG_ERR_ARG, "bad input: n must be in [1, 2^31)");
  int num_sms = 0;
  rc = device_of(&num_sms);
  if (rc) return rc;
  StreamHold sh;
  PBG_CUDA(cudaStreamCreateWithFlags(&sh.s, cudaStreamNonBlocking));
  DevMem d_text;
  PBG_CUDA(d_text.alloc(len - body));
  {
    Stage st;
    PBG_CUDA(st.init());
    Source src;
    src.mem = text;
    rc = to_device(src, body, len - body, d_text.as<char>(), st, sh.s);
    if (rc) return rc;
  }
  return parse_body(d_text.as<uint8_t>(), len - body, nm[0], nm[1], flags, num_sms, sh.s, out);
}

extern "C" int pbg_graph_load_adj(const char* path, uint32_t flags, pbg_graph** out) {
  if (!path || !out) return fail(PBG_ERR_ARG, "NULL argument");
  Fd fh;
  fh.fd = open(path, O_RDONLY);
  if (fh.fd < 0) return fail(PBG_ERR_ARG, std::string("unable to open file: ") + path);
  struct stat sb;
  if (fstat(fh.fd, &sb) != 0) return fail(PBG_ERR_ARG, "file is not readable");
  const uint64_t size = (uint64_t)sb.st_size;
  int num_sms = 0;
  int rc = device_of(&num_sms);
  if (rc) return rc;
  StreamHold sh;
  PBG_CUDA(cudaStreamCreateWithFlags(&sh.s, cudaStreamNonBlocking));
  DevMem d_text;
  uint64_t nm[2] = {0, 0}, body = 0;
  {
    Stage st;
    PBG_CUDA(st.init());
    Source src;
    src.fd = fh.fd;
    // the header from the first piece
    const uint64_t first = std::min<uint64_t>(size, STAGE_BYTES);
    if (!fill_part(src, st.h[0], 0, first)) return fail(PBG_ERR_ARG, "file read failed");
    rc = parse_header(st.h[0], first, ADJ_HEADER, nm, 2, &body);
    if (rc) return rc;
    PBG_CUDA(d_text.alloc(size - body));
    rc = to_device(src, body, size - body, d_text.as<char>(), st, sh.s);
    if (rc) return rc;
  }
  return parse_body(d_text.as<uint8_t>(), size - body, nm[0], nm[1], flags, num_sms, sh.s, out);
}

extern "C" int pbg_graph_write_adj(const pbg_graph* g, const char* path) {
  if (!g || !path) return fail(PBG_ERR_ARG, "NULL argument");
  File fh;
  fh.f = fopen(path, "wb");
  if (!fh.f) return fail(PBG_ERR_ARG, std::string("unable to open file: ") + path);
  Stage st;
  PBG_CUDA(st.init());
  // the layout of common/graphIO.h:79-104: header, n, m, n offsets, m edges
  if (fprintf(fh.f, "%s\n%u\n%llu\n", ADJ_HEADER, g->n, (unsigned long long)g->m) < 0)
    return fail(PBG_ERR_ARG, "file write failed");
  int rc = write_values(fh.f, g->d_offsets, g->n, false, st, g->stream);
  if (!rc) rc = write_values(fh.f, g->d_edges, g->m, false, st, g->stream);
  if (rc) return rc;
  if (fclose(fh.f) != 0) {
    fh.f = nullptr;
    return fail(PBG_ERR_ARG, "file close failed");
  }
  fh.f = nullptr;
  return PBG_OK;
}

extern "C" int pbg_write_seq_int(const int32_t* values, uint64_t count, const char* path) {
  if ((!values && count) || !path) return fail(PBG_ERR_ARG, "NULL argument");
  File fh;
  fh.f = fopen(path, "wb");
  if (!fh.f) return fail(PBG_ERR_ARG, std::string("unable to open file: ") + path);
  Stage st;
  PBG_CUDA(st.init());
  StreamHold sh;
  PBG_CUDA(cudaStreamCreateWithFlags(&sh.s, cudaStreamNonBlocking));
  if (fprintf(fh.f, "%s\n", SEQ_INT_HEADER) < 0) return fail(PBG_ERR_ARG, "file write failed");
  DevMem d;
  PBG_CUDA(d.alloc(sizeof(int32_t) * count));
  PBG_CUDA(cudaMemcpyAsync(d.p, values, sizeof(int32_t) * count, cudaMemcpyHostToDevice, sh.s));
  int rc = write_values(fh.f, d.as<uint32_t>(), count, true, st, sh.s);
  if (rc) return rc;
  if (fclose(fh.f) != 0) {
    fh.f = nullptr;
    return fail(PBG_ERR_ARG, "file close failed");
  }
  fh.f = nullptr;
  return PBG_OK;
}

extern "C" int pbg_graph_save_bin(const pbg_graph* g, const char* path) {
  if (!g || !path) return fail(PBG_ERR_ARG, "NULL argument");
  File fh;
  fh.f = fopen(path, "wb");
  if (!fh.f) return fail(PBG_ERR_ARG, std::string("unable to open file: ") + path);
  BinHeader h;
  memcpy(h.magic, BIN_MAGIC, 8);
  h.n = g->n;
  h.m = g->m;
  h.flags = g->flags & PBG_GRAPH_SYMMETRIC;
  h.reserved = 0;
  if (fwrite(&h, sizeof(h), 1, fh.f) != 1) return fail(PBG_ERR_ARG, "file write failed");
  Stage st;
  PBG_CUDA(st.init());
  int rc = device_to_file(fh.f, reinterpret_cast<const char*>(g->d_offsets), 4 * ((uint64_t)g->n + 1), st, g->stream);
  if (!rc) rc = device_to_file(fh.f, reinterpret_cast<const char*>(g->d_edges), 4 * g->m, st, g->stream);
  if (rc) return rc;
  if (fclose(fh.f) != 0) {
    fh.f = nullptr;
    return fail(PBG_ERR_ARG, "file close failed");
  }
  fh.f = nullptr;
  return PBG_OK;
}

extern "C" int pbg_graph_load_bin(const char* path, uint32_t flags, pbg_graph** out) {
  if (!path || !out) return fail(PBG_ERR_ARG, "NULL argument");
  Fd fh;
  fh.fd = open(path, O_RDONLY);
  if (fh.fd < 0) return fail(PBG_ERR_ARG, std::string("unable to open file: ") + path);
  Source src;
  src.fd = fh.fd;
  BinHeader h;
  if (!fill_part(src, reinterpret_cast<char*>(&h), 0, sizeof(h)) || memcmp(h.magic, BIN_MAGIC, 8) != 0)
    return fail(PBG_ERR_ARG, "not a binary CSR file (bad magic)");
  if (h.n == 0 || h.n > PBG_MAX_VERTICES || h.m > 0xFFFFFFFFull) return fail(PBG_ERR_ARG, "bad binary CSR header");
  struct stat sb;
  if (fstat(fh.fd, &sb) != 0) return fail(PBG_ERR_ARG, "file is not readable");
  if ((uint64_t)sb.st_size != sizeof(h) + 4 * (h.n + 1) + 4 * h.m)
    return fail(PBG_ERR_ARG, "binary CSR file size does not match its header");
  // the caller's flags; without a symmetry flag, the one the file was saved with
  const uint32_t fl = (flags & (PBG_GRAPH_SYMMETRIC | PBG_GRAPH_DETECT_SYMMETRIC)) ? flags : (flags | h.flags);
  pbg_graph* g = nullptr;
  int rc = new_handle((uint32_t)h.n, h.m, fl, &g);
  if (rc) return rc;
  {
    Stage st;
    cudaError_t e = st.init();
    if (e != cudaSuccess) {
      pbg_graph_free(g);
      return cuda_fail(e, "pinned staging");
    }
    rc = to_device(src, sizeof(h), 4 * (h.n + 1), reinterpret_cast<char*>(g->d_offsets), st, g->stream);
    if (!rc)
      rc = to_device(src, sizeof(h) + 4 * (h.n + 1), 4 * h.m, reinterpret_cast<char*>(g->d_edges), st, g->stream);
  }
  if (!rc) rc = finish_graph(g);
  if (rc) {
    pbg_graph_free(g);
    return rc;
  }
  *out = g;
  return PBG_OK;
}
