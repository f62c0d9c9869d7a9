// lists.cu -- device-resident list store, DPD metadata and JOBARC records.
//
// Replaces the reference's list I/O layer (acescore/getlst.F, putlst.F,
// aces_list_touch.F, acesutil/getall.F) and record store (getrec.F,
// putrec.F): lists are irrep-blocked column-major 2-D arrays held in device
// memory; GETLST/PUTLST copy column ranges between the list and the caller.
#include <cstdarg>
#include <cstring>

#include "common.cuh"

namespace acesb200 {

static thread_local char g_err[512] = "";
std::atomic<long long> g_launches{0};

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

State &state() {
  static State s;
  return s;
}

void *DeviceArena::alloc(size_t bytes) {
  bytes = (bytes + 255) & ~size_t(255);
  for (auto &c : chunks)
    if (c.size - c.used >= bytes) {
      void *p = c.base + c.used;
      c.used += bytes;
      return p;
    }
  size_t sz = bytes > chunk_bytes ? bytes : chunk_bytes;
  void *p = nullptr;
  if (dev_alloc((void **)&p, sz) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  chunks.push_back({(char *)p, sz, bytes});
  return p;
}

void DeviceArena::release() {
  for (auto &c : chunks) dev_free(c.base);
  chunks.clear();
}

size_t DeviceArena::total() const {
  size_t t = 0;
  for (auto &c : chunks) t += c.size;
  return t;
}

// Pair types 1..25 of acescore/aces_com_symloc.F (czTypes / szPacks).
PairType pair_type(int type) {
  static const char kP[25] = {'V', 'V', 'O', 'O', 'V', 'V', 'O', 'O', 'V', 'V', 'V', 'V', 'V',
                              'O', 'V', 'O', 'O', 'O', 'V', 'V', 'O', 'O', 'V', 'O', 'O'};
  static const char kQ[25] = {'V', 'V', 'O', 'O', 'V', 'V', 'O', 'O', 'O', 'O', 'O', 'O', 'V',
                              'O', 'V', 'V', 'V', 'V', 'V', 'V', 'O', 'O', 'V', 'O', 'V'};
  PairType t;
  t.p = kP[type - 1];
  t.q = kQ[type - 1];
  t.packing = type <= 4 ? 1 : (type <= 8 ? 2 : 0);
  return t;
}

long long pair_index(const SymInfo &s, int type, int hp, int p, int hq, int q) {
  PairType t = pair_type(type);
  int hpq = hp ^ hq;
  long long off = s.isymoff[hq][hpq][type - 1] - 1;
  int np = norb(s, t.p, hp);
  if (t.packing == 0) return off + p + (long long)q * np;
  if (hp < hq) return off + p + (long long)q * np;
  if (hp > hq) return -1;
  if (t.packing == 1) {
    if (p >= q) return -1;
    return off + p + (long long)q * (q - 1) / 2;
  }
  if (p > q) return -1;
  return off + p + (long long)q * (q + 1) / 2;
}

static int check_list(int irrep, int list, ListBlock **out) {
  State &st = state();
  if (irrep < 1 || irrep > 8 || list < 0 || list > 1000) {
    set_error("bad irrep %d or list %d", irrep, list);
    return ACES_ERR_ARG;
  }
  auto it = st.lists.find(list);
  if (it == st.lists.end() || it->second[irrep - 1].dev == nullptr) {
    set_error("list %d irrep %d not touched", list, irrep);
    return ACES_ERR_NOLIST;
  }
  *out = &it->second[irrep - 1];
  return ACES_OK;
}

static int copy_cols(double *ext, int first, int ncols, int irrep, int list, bool to_list,
                     cudaMemcpyKind kind, bool sync) {
  State &st = state();
  std::lock_guard<std::recursive_mutex> lk(st.mu);
  ListBlock *b;
  ACES_TRY(check_list(irrep, list, &b));
  if (ncols == 0) return ACES_OK;
  // acescore/getlst.F:52-90 bound assertions
  if (first < 1 || ncols < 0 || first - 1 + ncols > b->ncols) {
    set_error("columns %d..%d out of range (list %d irrep %d has %d)", first,
              first + ncols - 1, list, irrep, b->ncols);
    return ACES_ERR_ARG;
  }
  size_t bytes = (size_t)ncols * b->nrows * sizeof(double);
  double *lp = b->dev + (size_t)(first - 1) * b->nrows;
  if (bytes == 0) return ACES_OK;
  if (to_list)
    ACES_CUDA(cudaMemcpyAsync(lp, ext, bytes, kind, 0));
  else
    ACES_CUDA(cudaMemcpyAsync(ext, lp, bytes, kind, 0));
  if (sync) ACES_CUDA(cudaStreamSynchronize(0));
  return ACES_OK;
}

}  // namespace acesb200

using namespace acesb200;

extern "C" {

const char *aces_last_error(void) { return g_err; }

int aces_init(int device) {
  State &st = state();
  std::lock_guard<std::recursive_mutex> lk(st.mu);
  if (st.device >= 0) engine_reset();
  st.arena.release();
  st.lists.clear();
  st.isytyp.clear();
  st.records.clear();
  st.sym = SymInfo();
  ACES_CUDA(cudaSetDevice(device));
  st.device = device;
  return ACES_OK;
}

int aces_fin(void) {
  State &st = state();
  std::lock_guard<std::recursive_mutex> lk(st.mu);
  if (st.device >= 0) cudaDeviceSynchronize();
  engine_reset();
  st.arena.release();
  pool_trim();  // cached device blocks go back to the driver
  st.lists.clear();
  st.isytyp.clear();
  st.records.clear();
  st.sym = SymInfo();
  return ACES_OK;
}

int aces_sym_init(int nirrep, const int *pop, const int *vrt) {
  if (nirrep != 1 && nirrep != 2 && nirrep != 4 && nirrep != 8) {
    set_error("nirrep must be 1, 2, 4 or 8 (got %d)", nirrep);
    return ACES_ERR_ARG;
  }
  State &st = state();
  std::lock_guard<std::recursive_mutex> lk(st.mu);
  SymInfo &s = st.sym;
  s = SymInfo();
  s.nirrep = nirrep;
  for (int h = 0; h < nirrep; ++h) {
    if (pop[h] < 0 || vrt[h] < 0) return ACES_ERR_ARG;
    s.pop[h] = pop[h];
    s.vrt[h] = vrt[h];
  }
  // ISYMOFF: acescore/aces_com_symloc.F
  for (int type = 1; type <= 25; ++type) {
    PairType t = pair_type(type);
    for (int hpq = 0; hpq < nirrep; ++hpq) {
      int loc = 1;
      for (int hq = 0; hq < nirrep; ++hq) {
        int hp = hq ^ hpq;
        int np = norb(s, t.p, hp), nq = norb(s, t.q, hq);
        if (t.packing == 0) {
          s.isymoff[hq][hpq][type - 1] = loc;
          loc += np * nq;
        } else if (hp < hq) {
          s.isymoff[hq][hpq][type - 1] = loc;
          loc += np * nq;
        } else if (hp == hq) {
          s.isymoff[hq][hpq][type - 1] = loc;
          loc += t.packing == 1 ? np * (np - 1) / 2 : np * (np + 1) / 2;
        }
      }
      if (type <= 22) s.irpdpd[hpq][type - 1] = loc - 1;
    }
  }
  s.ready = true;
  return ACES_OK;
}

int aces_irpdpd(int irrep, int type) {
  const SymInfo &s = state().sym;
  if (!s.ready) return ACES_ERR_NOSYM;
  if (irrep < 1 || irrep > s.nirrep || type < 1 || type > 22) return ACES_ERR_ARG;
  return s.irpdpd[irrep - 1][type - 1];
}

int aces_isymoff(int irrep_q, int irrep_pq, int type) {
  const SymInfo &s = state().sym;
  if (!s.ready) return ACES_ERR_NOSYM;
  if (irrep_q < 1 || irrep_q > s.nirrep || irrep_pq < 1 || irrep_pq > s.nirrep || type < 1 ||
      type > 25)
    return ACES_ERR_ARG;
  return s.isymoff[irrep_q - 1][irrep_pq - 1][type - 1];
}

int aces_dirprd(int i, int j) {
  if (i < 1 || i > 8 || j < 1 || j > 8) return ACES_ERR_ARG;
  return ((i - 1) ^ (j - 1)) + 1;
}

int aces_list_touch(int ncols, int nrows, int irrep, int list, int nofrag) {
  (void)nofrag;
  State &st = state();
  std::lock_guard<std::recursive_mutex> lk(st.mu);
  if (irrep < 1 || irrep > 8 || list < 0 || list > 1000 || ncols < 0 || nrows < 0) {
    set_error("aces_list_touch: bad arguments (irrep %d list %d)", irrep, list);
    return ACES_ERR_ARG;
  }
  auto &v = st.lists[list];
  if (v.empty()) v.resize(8);
  ListBlock &b = v[irrep - 1];
  if (b.dev) {
    if (b.nrows == nrows && b.ncols == ncols) return ACES_OK;
    set_error("aces_list_touch: list %d irrep %d re-touched with %dx%d (was %dx%d)", list, irrep,
              nrows, ncols, b.nrows, b.ncols);
    return ACES_ERR_REDIM;
  }
  size_t bytes = (size_t)nrows * ncols * sizeof(double);
  void *p = st.arena.alloc(bytes ? bytes : 256);
  if (!p) {
    set_error("aces_list_touch: out of device memory for %zu bytes", bytes);
    return ACES_ERR_NOMEM;
  }
  if (bytes) ACES_CUDA(cudaMemset(p, 0, bytes));
  b.nrows = nrows;
  b.ncols = ncols;
  b.dev = (double *)p;
  return ACES_OK;
}

int aces_updmoi(int ncols, int nrows, int irrep, int list, int iarg1, int iarg2) {
  (void)iarg1;
  (void)iarg2;
  return aces_list_touch(ncols, nrows, irrep, list, 0);
}

int aces_inipck(int irrepx, int sytypl, int sytypr, int list, int iset) {
  State &st = state();
  std::lock_guard<std::recursive_mutex> lk(st.mu);
  const SymInfo &s = st.sym;
  if (!s.ready) return ACES_ERR_NOSYM;
  if (sytypl < 1 || sytypl > 22 || sytypr < 1 || sytypr > 22 || irrepx < 1 ||
      irrepx > s.nirrep) {
    set_error("aces_inipck: bad pair types %d/%d", sytypl, sytypr);
    return ACES_ERR_ARG;
  }
  for (int r = 1; r <= s.nirrep; ++r) {
    int l = aces_dirprd(r, irrepx);
    ACES_TRY(aces_list_touch(s.irpdpd[r - 1][sytypr - 1], s.irpdpd[l - 1][sytypl - 1], r, list, 0));
  }
  if (iset) st.isytyp[list == 0 ? 100 : list] = {sytypl, sytypr};
  return ACES_OK;
}

int aces_isytyp(int which, int list) {
  State &st = state();
  auto it = st.isytyp.find(list);
  if (it == st.isytyp.end() || (which != 1 && which != 2)) return ACES_ERR_ARG;
  return which == 1 ? it->second.first : it->second.second;
}

int aces_list_dims(int irrep, int list, int *ncols, int *nrows) {
  State &st = state();
  std::lock_guard<std::recursive_mutex> lk(st.mu);
  *ncols = 0;
  *nrows = 0;
  if (irrep < 1 || irrep > 8) return ACES_ERR_ARG;
  auto it = st.lists.find(list);
  if (it == st.lists.end()) return ACES_OK;
  *ncols = it->second[irrep - 1].ncols;
  *nrows = it->second[irrep - 1].nrows;
  return ACES_OK;
}

int aces_getlst(double *dst, int first, int ncols, int irrep, int list) {
  return copy_cols(dst, first, ncols, irrep, list, false, cudaMemcpyDeviceToHost, true);
}

int aces_putlst(const double *src, int first, int ncols, int irrep, int list) {
  return copy_cols(const_cast<double *>(src), first, ncols, irrep, list, true,
                   cudaMemcpyHostToDevice, true);
}

int aces_getlst_dev(double *dst, int first, int ncols, int irrep, int list) {
  return copy_cols(dst, first, ncols, irrep, list, false, cudaMemcpyDeviceToDevice, false);
}

int aces_putlst_dev(const double *src, int first, int ncols, int irrep, int list) {
  return copy_cols(const_cast<double *>(src), first, ncols, irrep, list, true,
                   cudaMemcpyDeviceToDevice, false);
}

static int getput_all(double *buf, long long len, int irrepx, int list, bool put) {
  State &st = state();
  std::lock_guard<std::recursive_mutex> lk(st.mu);
  const SymInfo &s = st.sym;
  if (!s.ready) return ACES_ERR_NOSYM;
  if (irrepx < 1 || irrepx > s.nirrep) return ACES_ERR_ARG;
  long long total = 0;
  for (int r = 1; r <= s.nirrep; ++r) {
    ListBlock *b;
    ACES_TRY(check_list(r, list, &b));
    total += (long long)b->nrows * b->ncols;
  }
  if (total != len) {
    set_error("GETALL/PUTALL length %lld != list %d size %lld", len, list, total);
    return ACES_ERR_ARG;
  }
  long long off = 0;
  for (int r = 1; r <= s.nirrep; ++r) {
    ListBlock *b;
    check_list(r, list, &b);
    size_t n = (size_t)b->nrows * b->ncols;
    if (n) {
      if (put)
        ACES_CUDA(cudaMemcpyAsync(b->dev, buf + off, n * 8, cudaMemcpyHostToDevice, 0));
      else
        ACES_CUDA(cudaMemcpyAsync(buf + off, b->dev, n * 8, cudaMemcpyDeviceToHost, 0));
    }
    off += n;
  }
  ACES_CUDA(cudaStreamSynchronize(0));
  return ACES_OK;
}

int aces_getall(double *dst, long long len, int irrepx, int list) {
  return getput_all(dst, len, irrepx, list, false);
}

int aces_putall(const double *src, long long len, int irrepx, int list) {
  return getput_all(const_cast<double *>(src), len, irrepx, list, true);
}

int aces_list_memset(int irrep, int list, int byte) {
  State &st = state();
  std::lock_guard<std::recursive_mutex> lk(st.mu);
  ListBlock *b;
  ACES_TRY(check_list(irrep, list, &b));
  size_t bytes = (size_t)b->nrows * b->ncols * 8;
  if (bytes) ACES_CUDA(cudaMemset(b->dev, byte & 0xff, bytes));
  return ACES_OK;
}

double *aces_list_devptr(int irrep, int list) {
  ListBlock *b;
  if (check_list(irrep, list, &b) != ACES_OK) return nullptr;
  return b->dev;
}

int aces_putrec(const char *label, long long nbytes, const void *buf) {
  if (!label || nbytes < 0 || (nbytes && !buf)) return ACES_ERR_ARG;
  State &st = state();
  std::lock_guard<std::recursive_mutex> lk(st.mu);
  std::vector<char> v((size_t)nbytes);
  if (nbytes) memcpy(v.data(), buf, (size_t)nbytes);
  st.records[label] = std::move(v);
  return ACES_OK;
}

int aces_getrec(const char *label, long long nbytes, void *buf) {
  if (!label || nbytes < 0) return ACES_ERR_ARG;
  State &st = state();
  std::lock_guard<std::recursive_mutex> lk(st.mu);
  auto it = st.records.find(label);
  if (it == st.records.end()) {
    set_error("record %s absent", label);
    return ACES_ERR_NOREC;
  }
  if ((size_t)nbytes > it->second.size()) {
    set_error("record %s holds %zu bytes, %lld requested", label, it->second.size(), nbytes);
    return ACES_ERR_ARG;
  }
  if (nbytes) memcpy(buf, it->second.data(), (size_t)nbytes);
  return ACES_OK;
}

long long aces_reclen(const char *label) {
  State &st = state();
  std::lock_guard<std::recursive_mutex> lk(st.mu);
  auto it = st.records.find(label ? label : "");
  if (it == st.records.end()) return ACES_ERR_NOREC;
  return (long long)it->second.size();
}

}  // extern "C"
