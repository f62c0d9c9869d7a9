// common.cuh -- shared state and helpers of the B200 CC engine.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/aces_b200.h"

namespace acesb200 {

void set_error(const char *fmt, ...);
// destroys the CC engine (amplitudes, intermediates, split caches) of this process
void engine_reset();

// caching device allocator (pool.cu): dev_free keeps the block for reuse by a
// later dev_alloc of the same size class on the same device; pool_trim
// returns every cached block to the driver
cudaError_t dev_alloc(void **ptr, size_t bytes);
void dev_free(void *ptr);
void pool_trim();

// number of kernels the library has launched (reported by the benchmarks)
extern std::atomic<long long> g_launches;
inline void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

#define ACES_CUDA(call)                                                        \
  do {                                                                         \
    cudaError_t _e = (call);                                                   \
    if (_e != cudaSuccess) {                                                   \
      ::acesb200::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,         \
                            cudaGetErrorString(_e));                           \
      return ACES_ERR_CUDA;                                                    \
    }                                                                          \
  } while (0)

#define ACES_TRY(call)                                                         \
  do {                                                                         \
    int _s = (call);                                                           \
    if (_s != ACES_OK) return _s;                                              \
  } while (0)

// Division of 32-bit indices below 2^31 by a run-time invariant divisor with
// a multiply-high, add and shift (Granlund and Montgomery, "Division by
// invariant integers using multiplication", PLDI 1994): with
// s = ceil(log2 d) and m = floor(2^32 (2^s - d) / d) + 1,
// n / d = (umulhi(n, m) + n) >> s for 0 <= n < 2^31.
struct FastDiv {
  unsigned d = 1, m = 1, s = 0;
  FastDiv() = default;
  explicit FastDiv(unsigned divisor) : d(divisor ? divisor : 1) {
    s = 0;
    while ((1ull << s) < d) ++s;
    m = (unsigned)(((1ull << 32) * ((1ull << s) - d)) / d + 1);
  }
  __host__ __device__ __forceinline__ unsigned div(unsigned n) const {
#ifdef __CUDA_ARCH__
    return (__umulhi(n, m) + n) >> s;
#else
    return (unsigned)((((unsigned long long)n * m) >> 32) + n) >> s;
#endif
  }
};

// One irrep block of a list: nrows x ncols doubles, column-major, on device.
struct ListBlock {
  int nrows = 0;
  int ncols = 0;
  double *dev = nullptr;
};

// Bump allocator over large device chunks: lists live until aces_fin, like
// the reference's single ICORE heap (acescore/aces_malloc.c).
struct DeviceArena {
  struct Chunk { char *base; size_t size; size_t used; };
  std::vector<Chunk> chunks;
  size_t chunk_bytes = size_t(256) << 20;
  void *alloc(size_t bytes);
  void release();
  size_t total() const;
};

struct SymInfo {
  int nirrep = 0;
  int pop[8] = {0};
  int vrt[8] = {0};
  int irpdpd[8][22] = {{0}};     // [irrep][type]
  int isymoff[8][8][25] = {{{0}}};  // [irp_q][irp_pq][type], 1-based
  bool ready = false;
};

struct State {
  std::recursive_mutex mu;
  int device = -1;
  SymInfo sym;
  std::map<int, std::vector<ListBlock>> lists;  // list id -> 8 irreps
  std::map<int, std::pair<int, int>> isytyp;    // list -> (left, right) type
  std::map<std::string, std::vector<char>> records;
  DeviceArena arena;
};

State &state();

// pair-type description: spins and occupied/virtual character of each index
struct PairType {
  char p, q;       // 'O' or 'V'
  int packing;     // 0 FULL, 1 PACK (p<q), 2 PCK2 (p<=q)
};
PairType pair_type(int type);   // type 1..25

// Orbital count of irrep h (0-based) for 'O'/'V' (RHF: alpha == beta).
inline int norb(const SymInfo &s, char c, int h) { return c == 'O' ? s.pop[h] : s.vrt[h]; }

// 0-based pair index (within the pairs of total irrep hpq) of local orbitals
// p (irrep hp) and q (irrep hq), or -1 when the pair is not stored
// (p >= q in a PACK block, p > q in a PCK2 block).
long long pair_index(const SymInfo &s, int type, int hp, int p, int hq, int q);

}  // namespace acesb200
