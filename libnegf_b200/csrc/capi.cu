// C-ABI of the B200 per-energy-point transport solve (include/negf_b200.h).
//
// Host side of the drop-in seam: a context owns one CUDA stream, the
// HBM-resident device descriptions (the counterpart of the H/S blocks and
// contact blocks libNEGF re-copies to the GPU at every energy point,
// src/iterative_gpu.F90:185-217), the persistent-kernel workspace and the
// per-call staging buffers.  Errors are returned as status codes; nothing
// here exits or traps (the reference stops on every error:
// src/ln_messages.F90:9-22, src/gpuroutines.cu:38-81).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/negf_b200.h"
#include "engine.cuh"
#include "mixed.cuh"
#include "small.cuh"
#include "ozaki.cuh"

using negf::DevDesc;

namespace {

struct DeviceRec {
  bool live = false;
  void* blob = nullptr;
  size_t bytes = 0;
  DevDesc desc{};
  int nbl = 0, ncont = 0, norb = 0, nmax = 0;
  int cblk[negf::kMaxCont] = {0};
  bool has_s = false;
  void* proj_tun = nullptr;    // device copies of the projections (owned)
  void* proj_dos = nullptr;
  int nldos = 0;
  // fingerprint of each contact's lead blocks (L, H00, H01, S00, S01): the surface
  // Green's function depends on nothing else, so a saved one is reused by any
  // device whose contact has the same lead
  uint64_t lead_hash[negf::kMaxCont] = {0};
};

// FNV-1a over a byte range, chained
uint64_t fnv1a(uint64_t h, const void* p, size_t n) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 0x100000001B3ull;
  }
  return h;
}

void free_projections(DeviceRec& r) {
  if (r.proj_tun) cudaFree(r.proj_tun);
  if (r.proj_dos) cudaFree(r.proj_dos);
  r.proj_tun = r.proj_dos = nullptr;
  r.desc.tun_mask = nullptr;
  r.desc.ldos_ptr = r.desc.ldos_idx = nullptr;
  r.desc.nldos = 0;
  r.nldos = 0;
}

}  // namespace

// Surface Green's function cache, the counterpart of libNEGF's
// surface_green_cache (src/ln_cache.F90; used by surface_green,
// src/contselfenergy.F90:146-167, 251-264).  The reference labels an entry
// by (k-point, energy point index, spin, contact); the batched calls here
// take energies, so an entry is labelled by (device, contact, E, eta, SGF
// tolerance, iteration cap).  Entries live in one device arena and are
// bump-allocated; when a launch's misses do not fit, they are computed
// without being stored, and the next launch that finds the arena full
// starts a new generation (all entries dropped).  Mode 1 loads what is
// cached and stores what is computed (ReadOldSGF = 0); mode 2 recomputes
// everything and overwrites (ReadOldSGF = 2).
struct SgfKey {
  int32_t dev, cont;
  uint64_t e, eta, tol;
  int32_t maxit;
  bool operator==(const SgfKey& o) const {
    return dev == o.dev && cont == o.cont && e == o.e && eta == o.eta && tol == o.tol && maxit == o.maxit;
  }
};
struct SgfKeyHash {
  size_t operator()(const SgfKey& k) const {
    uint64_t h = k.e * 0x9E3779B97F4A7C15ull ^ (k.eta + 0x632BE59BD9B4E019ull + ((uint64_t)k.dev << 32 | (uint32_t)k.cont));
    h ^= k.tol * 0xC2B2AE3D27D4EB4Full ^ (uint64_t)k.maxit;
    return (size_t)(h ^ (h >> 29));
  }
};
struct SgfCache {
  int mode = 0;
  double2* arena = nullptr;
  int64_t cap = 0, used = 0;   // complex elements
  std::unordered_map<SgfKey, int64_t, SgfKeyHash> map;
  int64_t hits = 0, misses = 0;
};

struct negf_b200_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  negf_b200_options opt{};
  std::string err;
  std::vector<DeviceRec> devs;
  DevDesc* d_descs = nullptr;
  size_t d_descs_cap = 0;
  bool descs_dirty = true;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  void* io = nullptr;
  size_t io_bytes = 0;
  void* pin = nullptr;     // pinned staging of large read-backs (ReadBack)
  size_t pin_bytes = 0;
  int sms = 0;
  bool trace = false;
  unsigned long long* d_trace = nullptr;
  SgfCache sgf;
  size_t ws_limit = 0;   // 0 = none
  uint64_t launches = 0; // kernels launched by solve calls (negf_b200_launch_count)
  std::mutex mu;
};

namespace {

int fail(negf_b200_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

int cuda_fail(negf_b200_ctx* ctx, cudaError_t e, const char* where) {
  return fail(ctx, NEGF_B200_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                        \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);            \
  } while (0)

int grow(negf_b200_ctx* ctx, void** p, size_t* cap, size_t need) {
  if (need <= *cap) return NEGF_B200_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc(p, need);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(ctx, NEGF_B200_ERR_NOMEM, "device allocation of " + std::to_string(need) + " bytes failed");
  }
  *cap = need;
  return NEGF_B200_OK;
}

// The device-to-host copies of one call's results.  A pageable destination
// makes the driver stage the copy through its own small pinned chunks, one
// synchronous round trip each (about 0.2 s for a 121 MB DOS array); results
// of 1 MiB and more therefore go through the context's pinned staging
// buffer at full link speed and are copied to the caller's memory after the
// stream synchronisation (finish()).  Without a staging buffer (cudaHostAlloc
// failed) they are copied directly.
struct ReadBack {
  static constexpr size_t kStageMin = 1 << 20;
  struct Item {
    void* dst;
    size_t off, bytes;
  };
  negf_b200_ctx* ctx;
  cudaStream_t s;
  char* pin = nullptr;
  size_t used = 0;
  std::vector<Item> staged;

  // reserve: the sum of the staged sizes of this call (one allocation, grown once)
  ReadBack(negf_b200_ctx* c, cudaStream_t st, size_t reserve) : ctx(c), s(st) {
    if (reserve == 0) return;
    if (ctx->pin_bytes < reserve) {
      if (ctx->pin) cudaFreeHost(ctx->pin);
      ctx->pin = nullptr;
      ctx->pin_bytes = 0;
      if (cudaHostAlloc(&ctx->pin, reserve, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        ctx->pin = nullptr;
        return;
      }
      ctx->pin_bytes = reserve;
    }
    pin = static_cast<char*>(ctx->pin);
  }
  static size_t staged_size(size_t bytes) { return bytes >= kStageMin ? (bytes + 255) / 256 * 256 : 0; }
  cudaError_t copy(void* dst, const void* src, size_t bytes) {
    if (!dst || bytes == 0) return cudaSuccess;
    if (pin && bytes >= kStageMin) {
      cudaError_t e = cudaMemcpyAsync(pin + used, src, bytes, cudaMemcpyDeviceToHost, s);
      staged.push_back({dst, used, bytes});
      used += staged_size(bytes);
      return e;
    }
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
  }
  void finish() {   // after the stream synchronisation
    for (const Item& it : staged) std::memcpy(it.dst, pin + it.off, it.bytes);
  }
};

int sync_descs(negf_b200_ctx* ctx) {
  if (!ctx->descs_dirty) return NEGF_B200_OK;
  size_t need = std::max<size_t>(1, ctx->devs.size()) * sizeof(DevDesc);
  int st = grow(ctx, reinterpret_cast<void**>(&ctx->d_descs), &ctx->d_descs_cap, need);
  if (st) return st;
  std::vector<DevDesc> h(ctx->devs.size());
  for (size_t i = 0; i < ctx->devs.size(); ++i) h[i] = ctx->devs[i].desc;
  if (!h.empty())
    CK(cudaMemcpy(ctx->d_descs, h.data(), h.size() * sizeof(DevDesc), cudaMemcpyHostToDevice));
  ctx->descs_dirty = false;
  return NEGF_B200_OK;
}

struct LaunchShape {
  int nmax = 0, nbl_max = 0, ncont_max = 0, norb_max = 0;
};

int shape_of(negf_b200_ctx* ctx, int npts, const int32_t* ids, LaunchShape& sh) {
  for (int p = 0; p < npts; ++p) {
    int id = ids ? ids[p] : -1;
    if (ids && (id < 0 || id >= (int)ctx->devs.size() || !ctx->devs[id].live))
      return fail(ctx, NEGF_B200_ERR_BAD_ARG, "point " + std::to_string(p) + ": unknown device id " +
                                                   std::to_string(id));
  }
  // host ids: the launch's own devices; device ids (the _dev calls): every live device
  std::vector<char> used;
  if (ids) {
    used.assign(ctx->devs.size(), 0);
    for (int p = 0; p < npts; ++p) used[ids[p]] = 1;
  }
  for (size_t i = 0; i < ctx->devs.size(); ++i) {
    const DeviceRec& r = ctx->devs[i];
    if (!r.live || (ids && !used[i])) continue;
    sh.nmax = std::max(sh.nmax, r.nmax);
    sh.nbl_max = std::max(sh.nbl_max, r.nbl);
    sh.ncont_max = std::max(sh.ncont_max, r.ncont);
    sh.norb_max = std::max(sh.norb_max, r.norb);
  }
  return NEGF_B200_OK;
}

int grid_for(negf_b200_ctx* ctx, int npts) {
  int per_sm = ctx->opt.ctas_per_sm > 0 ? ctx->opt.ctas_per_sm : 2;
  return std::max(1, std::min(npts, per_sm * ctx->sms));
}

// Runs one launch with device-resident inputs/outputs (all pointers device).
int run_device(negf_b200_ctx* ctx, negf::EngineArgs a, const LaunchShape& sh, cudaStream_t s) {
  if (sh.nmax > negf::kMaxOrder)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "block order " + std::to_string(sh.nmax) + " exceeds " +
                                                std::to_string(negf::kMaxOrder));
  int st = sync_descs(ctx);
  if (st) return st;
  int grid = grid_for(ctx, a.npts);
  const int64_t per = negf::engine_ws_elems(a.mode, sh.nbl_max, sh.ncont_max, sh.nmax);
  if (ctx->ws_limit > 0) {
    // fewer resident CTAs when the workspace would exceed the limit (the persistent
    // kernel still runs every point); not even one CTA: refuse
    const size_t per_bytes = (size_t)per * sizeof(double2);
    const size_t fit = ctx->ws_limit > 256 ? (ctx->ws_limit - 256) / per_bytes : 0;
    if (fit < 1)
      return fail(ctx, NEGF_B200_ERR_ADMISSION, "one CTA's workspace (" + std::to_string(per_bytes) +
                                                    " bytes) exceeds the workspace limit");
    grid = (int)std::min<size_t>(grid, fit);
  }
  // counter lives at the start of the workspace allocation
  const size_t need = 256 + (size_t)grid * per * sizeof(double2);
  st = grow(ctx, &ctx->ws, &ctx->ws_bytes, need);
  if (st) return st;
  a.counter = reinterpret_cast<int*>(ctx->ws);
  a.ws = reinterpret_cast<double2*>(reinterpret_cast<char*>(ctx->ws) + 256);
  a.ws_per_cta = per;
  a.Q = (int64_t)sh.nmax * sh.nmax;
  a.nmax = sh.nmax;
  a.nbl_max = sh.nbl_max;
  a.ncont_max = sh.ncont_max;
  a.devs = ctx->d_descs;
  a.trace = ctx->trace ? ctx->d_trace : nullptr;
  CK(cudaMemsetAsync(a.counter, 0, sizeof(int), s));
  cudaError_t e = negf::launch_engine(a, grid, s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "launch_engine");
  ++ctx->launches;
  return NEGF_B200_OK;
}

negf::EngineArgs base_args(negf_b200_ctx* ctx, int mode, int npts) {
  negf::EngineArgs a;
  std::memset(&a, 0, sizeof(a));
  a.mode = mode;
  a.npts = npts;
  a.sgf_tol = ctx->opt.sgf_tol;
  a.sgf_max_iter = ctx->opt.sgf_max_iter;
  a.eps = ctx->opt.eps_drop;
  a.scba_niter = ctx->opt.scba_niter;
  a.scba_tol = ctx->opt.scba_tol;
  a.scba_mix = ctx->opt.scba_mix;
  a.scba_rule = ctx->opt.scba_rule;
  return a;
}

int first_status(const int32_t* status, int npts) {
  for (int p = 0; p < npts; ++p)
    if (status[p] != NEGF_B200_OK) return status[p];
  return NEGF_B200_OK;
}

// Staging area carve-out on ctx->io
struct Carve {
  char* base;
  size_t off = 0;
  template <class T>
  T* take(size_t n) {
    off = (off + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base + off);
    off += n * sizeof(T);
    return p;
  }
};

uint64_t bits_of(double x) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  return u;
}

// Per point and contact: where to read gs from (hit) and where to store the
// computed one (miss with room), as arena offsets or -1.
void plan_sgf(negf_b200_ctx* ctx, int npts, const int32_t* ids, const double* E, double eta, int ncont_max,
              std::vector<int64_t>& in, std::vector<int64_t>& out) {
  SgfCache& c = ctx->sgf;
  in.assign((size_t)npts * ncont_max, -1);
  out.assign((size_t)npts * ncont_max, -1);
  // a new generation when the arena is full
  int64_t need = 0;
  for (int p = 0; p < npts; ++p) {
    const DeviceRec& r = ctx->devs[ids[p]];
    for (int k = 0; k < r.ncont; ++k) need += (int64_t)r.desc.L[k] * r.desc.L[k];
  }
  if (c.used > 0 && c.used + need > c.cap) {
    bool all_hit = true;
    for (int p = 0; p < npts && all_hit; ++p) {
      const DeviceRec& r = ctx->devs[ids[p]];
      for (int k = 0; k < r.ncont; ++k) {
        SgfKey key{ids[p], k, bits_of(E[p]), bits_of(eta), bits_of(ctx->opt.sgf_tol), ctx->opt.sgf_max_iter};
        if (!c.map.count(key)) { all_hit = false; break; }
      }
    }
    if (!all_hit) {
      c.map.clear();
      c.used = 0;
    }
  }
  std::unordered_map<SgfKey, int64_t, SgfKeyHash> fresh;   // stored by this launch: not readable in it
  for (int p = 0; p < npts; ++p) {
    const DeviceRec& r = ctx->devs[ids[p]];
    for (int k = 0; k < r.ncont; ++k) {
      const int64_t L2 = (int64_t)r.desc.L[k] * r.desc.L[k];
      SgfKey key{ids[p], k, bits_of(E[p]), bits_of(eta), bits_of(ctx->opt.sgf_tol), ctx->opt.sgf_max_iter};
      const size_t q = (size_t)p * ncont_max + k;
      auto it = c.map.find(key);
      if (c.mode == 1 && it != c.map.end() && !fresh.count(key)) {
        in[q] = it->second;
        ++c.hits;
        continue;
      }
      ++c.misses;
      if (fresh.count(key)) continue;                       // twice in one launch: compute, store once
      int64_t off = -1;
      if (it != c.map.end()) {
        off = it->second;                                   // refresh in place
      } else if (c.used + L2 <= c.cap) {
        off = c.used;
        c.used += (L2 + 15) & ~int64_t(15);
        c.map[key] = off;
      }
      if (off >= 0) {
        out[q] = off;
        fresh[key] = off;
      }
    }
  }
}

void drop_sgf_of(negf_b200_ctx* ctx, int dev) {
  for (auto it = ctx->sgf.map.begin(); it != ctx->sgf.map.end();)
    it = (it->first.dev == dev) ? ctx->sgf.map.erase(it) : std::next(it);
}

}  // namespace

extern "C" {

void negf_b200_default_options(negf_b200_options* o) {
  if (!o) return;
  o->sgf_tol = 1e-9;
  o->sgf_max_iter = 300;
  o->eps_drop = 0.0;
  o->scba_tol = 1e-7;
  o->scba_niter = 0;
  o->precision = 0;
  o->ctas_per_sm = 0;
  o->scba_mix = 1.0;
  o->scba_rule = 0;
  o->schedule = 0;
}

const char* negf_b200_version(void) { return "negf_b200 0.1 (sm_100a, complex FP64)"; }

int negf_b200_ctx_create(int32_t cuda_device, negf_b200_ctx** out) {
  if (!out) return NEGF_B200_ERR_BAD_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return NEGF_B200_ERR_NO_GPU;
  }
  if (cuda_device < 0 || cuda_device >= ndev) return NEGF_B200_ERR_BAD_ARG;
  negf_b200_ctx* ctx = new negf_b200_ctx();
  ctx->device = cuda_device;
  negf_b200_default_options(&ctx->opt);
  cudaError_t e = cudaSetDevice(cuda_device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, cuda_device);
  if (e != cudaSuccess) {
    delete ctx;
    return NEGF_B200_ERR_CUDA;
  }
  *out = ctx;
  return NEGF_B200_OK;
}

int negf_b200_ctx_destroy(negf_b200_ctx* ctx) {
  if (!ctx) return NEGF_B200_ERR_BAD_ARG;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& r : ctx->devs) {
    if (r.blob) cudaFree(r.blob);
    free_projections(r);
  }
  if (ctx->d_descs) cudaFree(ctx->d_descs);
  if (ctx->ws) cudaFree(ctx->ws);
  if (ctx->io) cudaFree(ctx->io);
  if (ctx->pin) cudaFreeHost(ctx->pin);
  if (ctx->d_trace) cudaFree(ctx->d_trace);
  if (ctx->sgf.arena) cudaFree(ctx->sgf.arena);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return NEGF_B200_OK;
}

int negf_b200_set_options(negf_b200_ctx* ctx, const negf_b200_options* o) {
  if (!ctx || !o) return NEGF_B200_ERR_BAD_ARG;
  if (o->sgf_tol <= 0.0 || o->sgf_max_iter < 1 || o->scba_niter < 0 || o->ctas_per_sm < 0 ||
      o->ctas_per_sm > 2)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "invalid options");
  if (o->precision != 0 && o->precision != 1 && (o->precision < negf::kOzMinSlices || o->precision > negf::kOzMaxSlices))
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "precision must be 0 (FP64), 1 or 4..8 (int8 digits of the mixed form)");
  if (!(o->scba_mix > 0.0 && o->scba_mix <= 1.0) || (o->scba_rule != 0 && o->scba_rule != 1))
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "scba_mix must be in (0, 1] and scba_rule 0 or 1");
  if (o->schedule < 0 || o->schedule > 2)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "schedule must be 0 (auto), 1 (engine) or 2 (lock step)");
  ctx->opt = *o;
  return NEGF_B200_OK;
}

const char* negf_b200_last_error(const negf_b200_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

int negf_b200_launch_count(negf_b200_ctx* ctx, uint64_t* count) {
  if (!ctx || !count) return NEGF_B200_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  *count = ctx->launches;
  return NEGF_B200_OK;
}

namespace {
// The block arrays of `dv` may be host or device memory (copies with
// cudaMemcpyDefault); pl_size, cblk and lead_size are host arrays.
int upload_impl(negf_b200_ctx* ctx, const negf_b200_device* dv, int32_t* device_id) {
  const int nbl = dv->nbl, ncont = dv->ncont;
  if (nbl < 1 || !dv->pl_size || !dv->h_diag || (nbl > 1 && (!dv->h_upper || !dv->h_lower)))
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "device needs nbl >= 1 and H blocks");
  if (ncont < 1 || ncont > negf::kMaxCont || !dv->cblk || !dv->lead_size || !dv->lead_h00 || !dv->lead_h01 ||
      !dv->hmc)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "device needs 1..10 contacts with lead and coupling blocks");
  const bool has_s = dv->s_diag != nullptr;
  if (has_s && nbl > 1 && (!dv->s_upper || !dv->s_lower))
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "S blocks must be all given or all NULL");
  std::vector<int32_t> pl(dv->pl_size, dv->pl_size + nbl), pstart(nbl);
  std::vector<int64_t> od(nbl), oo(std::max(1, nbl - 1));
  int64_t nd = 0, no = 0;
  int norb = 0, nmax = 0;
  for (int i = 0; i < nbl; ++i) {
    if (pl[i] < 1) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "PL size must be >= 1");
    pstart[i] = norb;
    norb += pl[i];
    nmax = std::max(nmax, pl[i]);
    od[i] = nd;
    nd += (int64_t)pl[i] * pl[i];
    if (i + 1 < nbl) {
      oo[i] = no;
      no += (int64_t)pl[i] * pl[i + 1];
    }
  }
  int64_t nl = 0, nm = 0, nsf = 0;
  std::vector<int64_t> olead(ncont), omc(ncont), osurf(ncont, 0);
  std::vector<int> surf(ncont, 0);
  for (int c = 0; c < ncont; ++c) {
    const int cb = dv->cblk[c], L = dv->lead_size[c];
    if (cb < 1 || cb > nbl || L < 1)
      return fail(ctx, NEGF_B200_ERR_BAD_ARG, "contact " + std::to_string(c + 1) + ": bad cblk or lead size");
    surf[c] = dv->surf_size ? dv->surf_size[c] : 0;
    if (surf[c] < 0 || (surf[c] > 0 && !dv->lead_hs))
      return fail(ctx, NEGF_B200_ERR_BAD_ARG, "contact " + std::to_string(c + 1) + ": bad surface block");
    const int ngs = L + surf[c];   // orbitals of the contact the device couples to (Surf + PL1)
    nmax = std::max(nmax, ngs);
    olead[c] = nl;
    nl += (int64_t)L * L;
    omc[c] = nm;
    nm += (int64_t)pl[cb - 1] * ngs;
    if (surf[c] > 0) {
      osurf[c] = nsf;
      nsf += (int64_t)ngs * ngs;
    }
  }
  if (nmax > negf::kMaxOrder)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "block order above " + std::to_string(negf::kMaxOrder));
  // blob layout (complex elements): hd sd | hu hl su sl | h00 h01 s00 s01 | hmc smc | ints
  const int64_t ns = has_s ? 1 : 0;
  const int64_t has00 = dv->lead_s00 ? 1 : 0, has01 = dv->lead_s01 ? 1 : 0, hasmc = dv->smc ? 1 : 0;
  const int64_t hasss = (nsf > 0 && dv->lead_ss) ? 1 : 0;
  int64_t elems = nd * (1 + ns) + no * (2 + 2 * ns) + nl * (2 + has00 + has01) + nm * (1 + hasmc) +
                  nsf * (1 + hasss);
  size_t bytes = (size_t)elems * 16 + (size_t)nbl * (4 + 4 + 8) + (size_t)std::max(1, nbl - 1) * 8 + 64;
  int st;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  void* blob = nullptr;
  if (cudaMalloc(&blob, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, NEGF_B200_ERR_NOMEM, "device allocation of the device description failed");
  }
  char* b = reinterpret_cast<char*>(blob);
  size_t off = 0;
  cudaError_t perr = cudaSuccess;
  // synchronous copies on the legacy stream: no device-wide synchronisation, so an
  // upload does not wait for launches running on other (non-blocking) streams
  auto put = [&](const void* src, size_t nbytes) -> void* {
    void* dst = b + off;
    off += (nbytes + 15) & ~size_t(15);
    if (src && nbytes) {
      cudaError_t ce = cudaMemcpy(dst, src, nbytes, cudaMemcpyDefault);
      if (ce != cudaSuccess) perr = ce;
    }
    return dst;
  };
  DevDesc d{};
  d.nbl = nbl; d.ncont = ncont; d.norb = norb; d.has_s = has_s ? 1 : 0;
  d.has_s00 = (int)has00; d.has_s01 = (int)has01; d.has_smc = (int)hasmc;
  d.hd = (const double2*)put(dv->h_diag, nd * 16);
  d.sd = has_s ? (const double2*)put(dv->s_diag, nd * 16) : nullptr;
  d.hu = (const double2*)put(nbl > 1 ? dv->h_upper : nullptr, no * 16);
  d.hl = (const double2*)put(nbl > 1 ? dv->h_lower : nullptr, no * 16);
  d.su = has_s ? (const double2*)put(nbl > 1 ? dv->s_upper : nullptr, no * 16) : nullptr;
  d.sl = has_s ? (const double2*)put(nbl > 1 ? dv->s_lower : nullptr, no * 16) : nullptr;
  d.h00 = (const double2*)put(dv->lead_h00, nl * 16);
  d.h01 = (const double2*)put(dv->lead_h01, nl * 16);
  d.s00 = has00 ? (const double2*)put(dv->lead_s00, nl * 16) : nullptr;
  d.s01 = has01 ? (const double2*)put(dv->lead_s01, nl * 16) : nullptr;
  d.hmc = (const double2*)put(dv->hmc, nm * 16);
  d.smc = hasmc ? (const double2*)put(dv->smc, nm * 16) : nullptr;
  d.hs = nsf > 0 ? (const double2*)put(dv->lead_hs, nsf * 16) : nullptr;
  d.ss = hasss ? (const double2*)put(dv->lead_ss, nsf * 16) : nullptr;
  d.has_ss = (int)hasss;
  d.pl = (const int*)put(pl.data(), nbl * 4);
  d.pstart = (const int*)put(pstart.data(), nbl * 4);
  d.od = (const int64_t*)put(od.data(), nbl * 8);
  d.oo = (const int64_t*)put(oo.data(), oo.size() * 8);
  for (int c = 0; c < ncont; ++c) {
    d.cblk[c] = dv->cblk[c];
    d.L[c] = dv->lead_size[c];
    d.olead[c] = olead[c];
    d.omc[c] = omc[c];
    d.surf[c] = surf[c];
    d.osurf[c] = osurf[c];
  }
  if (perr != cudaSuccess || off > bytes) {
    cudaGetLastError();
    cudaFree(blob);
    return fail(ctx, NEGF_B200_ERR_CUDA, "upload of the device description failed");
  }
  DeviceRec r;
  r.live = true; r.blob = blob; r.bytes = bytes; r.desc = d;
  r.nbl = nbl; r.ncont = ncont; r.norb = norb; r.nmax = nmax; r.has_s = has_s;
  for (int c = 0; c < ncont; ++c) {
    r.cblk[c] = dv->cblk[c];
    const int L = dv->lead_size[c];
    const size_t nb = (size_t)L * L * 16;
    std::vector<char> tmp(nb);
    auto blk = [&](const double2* p) {   // the uploaded copy: host and device sources alike
      if (cudaMemcpy(tmp.data(), p + olead[c], nb, cudaMemcpyDeviceToHost) != cudaSuccess) perr = cudaErrorUnknown;
      return tmp.data();
    };
    uint64_t h = fnv1a(0xCBF29CE484222325ull, &L, sizeof(L));
    h = fnv1a(h, blk(d.h00), nb);
    h = fnv1a(h, blk(d.h01), nb);
    const int32_t f00 = has00 ? 1 : 0, f01 = has01 ? 1 : 0;
    h = fnv1a(h, &f00, 4);
    if (has00) h = fnv1a(h, blk(d.s00), nb);
    h = fnv1a(h, &f01, 4);
    if (has01) h = fnv1a(h, blk(d.s01), nb);
    r.lead_hash[c] = h;
  }
  if (perr != cudaSuccess) {
    cudaGetLastError();
    cudaFree(blob);
    return fail(ctx, NEGF_B200_ERR_CUDA, "upload of the device description failed");
  }
  int id = -1;
  for (size_t i = 0; i < ctx->devs.size(); ++i)
    if (!ctx->devs[i].live) { id = (int)i; break; }
  if (id < 0) { id = (int)ctx->devs.size(); ctx->devs.push_back(r); } else ctx->devs[id] = r;
  ctx->descs_dirty = true;
  *device_id = id;
  (void)st;
  return NEGF_B200_OK;
}
}  // namespace

int negf_b200_upload_device(negf_b200_ctx* ctx, const negf_b200_device* dv, int32_t* device_id) {
  if (!ctx || !dv || !device_id) return NEGF_B200_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return upload_impl(ctx, dv, device_id);
}

int negf_b200_upload_csr(negf_b200_ctx* ctx, int32_t nrow, int32_t nnz, const int32_t* rowptr, const int32_t* colind,
                         const double* h_vals, const double* s_vals, int32_t npl, const int32_t* plend,
                         int32_t ncont, const int32_t* cblk, const int32_t* surfstart, const int32_t* surfend,
                         const int32_t* contend, int32_t* device_id) {
  if (!ctx || !device_id) return NEGF_B200_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (nrow < 1 || nnz < 0 || !rowptr || (nnz > 0 && (!colind || !h_vals)) || npl < 1 || !plend || ncont < 1 ||
      ncont > negf::kMaxCont || !cblk || !surfstart || !surfend || !contend)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "bad CSR or structure arrays");
  if (rowptr[0] != 1 || rowptr[nrow] != nnz + 1)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "rowptr must be 1-based with rowptr(nrow+1) = nnz + 1");
  // create_TStruct: PLs from plend, contacts from surfstart / surfend / contend
  std::vector<int32_t> pl(npl), plstart(npl + 1, 0), L(ncont);
  std::vector<int64_t> od(npl), oo(std::max(1, npl - 1));
  int64_t nd = 0, no = 0, nl = 0, nm = 0;
  for (int i = 0; i < npl; ++i) {
    plstart[i + 1] = plend[i];
    pl[i] = plend[i] - plstart[i];
    if (pl[i] < 1) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "plend must increase");
    od[i] = nd;
    nd += (int64_t)pl[i] * pl[i];
  }
  for (int i = 0; i + 1 < npl; ++i) {
    oo[i] = no;
    no += (int64_t)pl[i] * pl[i + 1];
  }
  negf::CsrScatter a{};
  a.nrow = nrow; a.nnz = nnz; a.ndev = plend[npl - 1]; a.npl = npl; a.ncont = ncont;
  for (int c = 0; c < ncont; ++c) {
    const int ncdim = contend[c] - surfstart[c] + 1;
    if (surfend[c] != surfstart[c] - 1)
      return fail(ctx, NEGF_B200_ERR_BAD_ARG, "contact " + std::to_string(c + 1) +
                                                  ": surface blocks (surfdim > 0) are not supported");
    if (ncdim < 2 || ncdim % 2 || contend[c] > nrow || surfstart[c] <= a.ndev || cblk[c] < 1 || cblk[c] > npl)
      return fail(ctx, NEGF_B200_ERR_BAD_ARG, "contact " + std::to_string(c + 1) + ": bad extent or cblk");
    L[c] = ncdim / 2;
    a.j0[c] = surfstart[c] - 1; a.L[c] = L[c]; a.cb[c] = cblk[c];
    a.olead[c] = nl; nl += (int64_t)L[c] * L[c];
    a.omc[c] = nm; nm += (int64_t)pl[cblk[c] - 1] * L[c];
  }
  const bool has_s = s_vals != nullptr;
  const int64_t ns = has_s ? 2 : 1;
  // one scratch allocation: staging blocks, then the CSR and index copies
  const int64_t blk_elems = ns * (nd + 2 * no + 2 * nl + nm);
  size_t off = 0;
  auto carve = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~size_t(255); return o; };
  const size_t o_blk = carve((size_t)blk_elems * 16), o_rp = carve((size_t)(nrow + 1) * 4),
               o_ci = carve((size_t)std::max(nnz, 1) * 4), o_hv = carve((size_t)std::max(nnz, 1) * 16),
               o_sv = carve(has_s ? (size_t)std::max(nnz, 1) * 16 : 0), o_ps = carve((size_t)(npl + 1) * 4),
               o_od = carve((size_t)npl * 8), o_oo = carve(oo.size() * 8), o_bad = carve(4);
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  char* tmp = nullptr;
  if (cudaMalloc(&tmp, off) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, NEGF_B200_ERR_NOMEM, "device allocation of the CSR staging failed");
  }
  cudaStream_t s = ctx->stream;
  double2* blk = reinterpret_cast<double2*>(tmp + o_blk);
  double2* p = blk;
  auto take = [&](int64_t n) { double2* q = p; p += n; return q; };
  a.hd = take(nd); a.hu = take(no); a.hl = take(no); a.h00 = take(nl); a.h01 = take(nl); a.hmc = take(nm);
  if (has_s) { a.sd = take(nd); a.su = take(no); a.sl = take(no); a.s00 = take(nl); a.s01 = take(nl); a.smc = take(nm); }
  a.rowptr = reinterpret_cast<const int*>(tmp + o_rp);
  a.colind = reinterpret_cast<const int*>(tmp + o_ci);
  a.hv = reinterpret_cast<const double2*>(tmp + o_hv);
  a.sv = has_s ? reinterpret_cast<const double2*>(tmp + o_sv) : nullptr;
  a.plstart = reinterpret_cast<const int*>(tmp + o_ps);
  a.od = reinterpret_cast<const int64_t*>(tmp + o_od);
  a.oo = reinterpret_cast<const int64_t*>(tmp + o_oo);
  a.bad = reinterpret_cast<int*>(tmp + o_bad);
  cudaError_t e = cudaMemsetAsync(blk, 0, (size_t)blk_elems * 16, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(a.bad, 0, 4, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(tmp + o_rp, rowptr, (size_t)(nrow + 1) * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && nnz > 0) e = cudaMemcpyAsync(tmp + o_ci, colind, (size_t)nnz * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && nnz > 0) e = cudaMemcpyAsync(tmp + o_hv, h_vals, (size_t)nnz * 16, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && has_s && nnz > 0)
    e = cudaMemcpyAsync(tmp + o_sv, s_vals, (size_t)nnz * 16, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(tmp + o_ps, plstart.data(), (size_t)(npl + 1) * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(tmp + o_od, od.data(), (size_t)npl * 8, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(tmp + o_oo, oo.data(), oo.size() * 8, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = negf::launch_csr_scatter(a, s);
  int bad = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, a.bad, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    cudaFree(tmp);
    return cuda_fail(ctx, e, "CSR extraction");
  }
  if (bad) {
    cudaFree(tmp);
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "CSR index outside the matrix or rowptr not monotone");
  }
  negf_b200_device dv{};
  dv.nbl = npl; dv.pl_size = pl.data(); dv.ncont = ncont; dv.cblk = cblk; dv.lead_size = L.data();
  auto dp = [](const double2* q) { return reinterpret_cast<const double*>(q); };
  dv.h_diag = dp(a.hd); dv.h_upper = dp(a.hu); dv.h_lower = dp(a.hl);
  dv.lead_h00 = dp(a.h00); dv.lead_h01 = dp(a.h01); dv.hmc = dp(a.hmc);
  if (has_s) {
    dv.s_diag = dp(a.sd); dv.s_upper = dp(a.su); dv.s_lower = dp(a.sl);
    dv.lead_s00 = dp(a.s00); dv.lead_s01 = dp(a.s01); dv.smc = dp(a.smc);
  }
  const int st = upload_impl(ctx, &dv, device_id);
  cudaFree(tmp);
  return st;
}

int negf_b200_release_device(negf_b200_ctx* ctx, int32_t id) {
  if (!ctx) return NEGF_B200_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (id < 0 || id >= (int)ctx->devs.size() || !ctx->devs[id].live)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "unknown device id");
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->devs[id].blob);
  free_projections(ctx->devs[id]);
  drop_sgf_of(ctx, id);
  ctx->devs[id] = DeviceRec();
  ctx->descs_dirty = true;
  return NEGF_B200_OK;
}

int negf_b200_device_bytes(const negf_b200_ctx* ctx, int32_t id, size_t* bytes) {
  if (!ctx || !bytes || id < 0 || id >= (int)ctx->devs.size() || !ctx->devs[id].live)
    return NEGF_B200_ERR_BAD_ARG;
  *bytes = ctx->devs[id].bytes;
  return NEGF_B200_OK;
}

int negf_b200_set_tun_proj(negf_b200_ctx* ctx, int32_t id, int32_t nidx, const int32_t* idx) {
  if (!ctx) return NEGF_B200_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (id < 0 || id >= (int)ctx->devs.size() || !ctx->devs[id].live)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "unknown device id");
  if (nidx < 0 || (nidx > 0 && !idx)) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "bad tun_proj index array");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  cudaStreamSynchronize(ctx->stream);
  DeviceRec& r = ctx->devs[id];
  if (r.proj_tun) cudaFree(r.proj_tun);
  r.proj_tun = nullptr;
  r.desc.tun_mask = nullptr;
  ctx->descs_dirty = true;
  if (nidx == 0) return NEGF_B200_OK;
  // get_tun_mask (src/iterative_cpu.F90:586-618): indices outside the device are ignored
  std::vector<unsigned char> mask(r.norb, 0);
  for (int q = 0; q < nidx; ++q)
    if (idx[q] >= 1 && idx[q] <= r.norb) mask[idx[q] - 1] = 1;
  if (cudaMalloc(&r.proj_tun, r.norb) != cudaSuccess) {
    cudaGetLastError();
    r.proj_tun = nullptr;
    return fail(ctx, NEGF_B200_ERR_NOMEM, "device allocation of the tun_proj mask failed");
  }
  CK(cudaMemcpy(r.proj_tun, mask.data(), r.norb, cudaMemcpyHostToDevice));
  r.desc.tun_mask = reinterpret_cast<const unsigned char*>(r.proj_tun);
  return NEGF_B200_OK;
}

int negf_b200_set_dos_proj(negf_b200_ctx* ctx, int32_t id, int32_t nsets, const int32_t* set_ptr,
                           const int32_t* set_idx) {
  if (!ctx) return NEGF_B200_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (id < 0 || id >= (int)ctx->devs.size() || !ctx->devs[id].live)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "unknown device id");
  if (nsets < 0 || (nsets > 0 && !set_ptr)) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "bad dos_proj arrays");
  const int nidx = nsets > 0 ? set_ptr[nsets] : 0;
  if (nsets > 0) {
    if (set_ptr[0] != 0 || (nidx > 0 && !set_idx)) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "bad dos_proj arrays");
    for (int k = 0; k < nsets; ++k)
      if (set_ptr[k + 1] < set_ptr[k]) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "dos_proj set_ptr must not decrease");
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  cudaStreamSynchronize(ctx->stream);
  DeviceRec& r = ctx->devs[id];
  if (r.proj_dos) cudaFree(r.proj_dos);
  r.proj_dos = nullptr;
  r.desc.ldos_ptr = r.desc.ldos_idx = nullptr;
  r.desc.nldos = 0;
  r.nldos = 0;
  ctx->descs_dirty = true;
  if (nsets == 0) return NEGF_B200_OK;
  const size_t bytes = (size_t)(nsets + 1 + std::max(1, nidx)) * 4;
  if (cudaMalloc(&r.proj_dos, bytes) != cudaSuccess) {
    cudaGetLastError();
    r.proj_dos = nullptr;
    return fail(ctx, NEGF_B200_ERR_NOMEM, "device allocation of the dos_proj sets failed");
  }
  int* d = reinterpret_cast<int*>(r.proj_dos);
  CK(cudaMemcpy(d, set_ptr, (size_t)(nsets + 1) * 4, cudaMemcpyHostToDevice));
  if (nidx > 0) CK(cudaMemcpy(d + nsets + 1, set_idx, (size_t)nidx * 4, cudaMemcpyHostToDevice));
  r.desc.ldos_ptr = d;
  r.desc.ldos_idx = d + nsets + 1;
  r.desc.nldos = nsets;
  r.nldos = nsets;
  return NEGF_B200_OK;
}

int negf_b200_set_sgf_cache(negf_b200_ctx* ctx, int32_t mode, size_t bytes) {
  if (!ctx || mode < 0 || mode > 2) return NEGF_B200_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  cudaStreamSynchronize(ctx->stream);
  SgfCache& c = ctx->sgf;
  const int64_t cap = (int64_t)(bytes / sizeof(double2));
  if (mode == 0 || cap != c.cap) {
    if (c.arena) cudaFree(c.arena);
    c.arena = nullptr;
    c.cap = c.used = 0;
    c.map.clear();
  }
  c.mode = 0;
  if (mode == 0) return NEGF_B200_OK;
  if (cap < 1) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "the SGF cache needs a positive size");
  if (!c.arena) {
    if (cudaMalloc(&c.arena, (size_t)cap * sizeof(double2)) != cudaSuccess) {
      cudaGetLastError();
      c.arena = nullptr;
      c.cap = 0;
      return fail(ctx, NEGF_B200_ERR_NOMEM, "device allocation of the SGF cache failed");
    }
    c.cap = cap;
  }
  c.mode = mode;
  return NEGF_B200_OK;
}

int negf_b200_set_workspace_limit(negf_b200_ctx* ctx, size_t bytes) {
  if (!ctx) return NEGF_B200_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->ws_limit = bytes;
  if (bytes > 0 && ctx->ws_bytes > bytes) {   // give back a larger arena now
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->ws);
    ctx->ws = nullptr;
    ctx->ws_bytes = 0;
  }
  return NEGF_B200_OK;
}

// File layout (little-endian): "NEGFSGF1", int64 count, then per entry
// uint64 lead fingerprint, int32 L, int32 maxit, uint64 bits of E, eta, tol,
// L*L complex128 (column-major) values.
namespace {
const char kSgfMagic[8] = {'N', 'E', 'G', 'F', 'S', 'G', 'F', '1'};
struct SgfFileEntry {
  uint64_t hash;
  int32_t L, maxit;
  uint64_t e, eta, tol;
};
}  // namespace

int negf_b200_sgf_cache_save(negf_b200_ctx* ctx, const char* path, int64_t* entries) {
  if (!ctx || !path) return NEGF_B200_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream));
  const SgfCache& c = ctx->sgf;
  std::vector<double2> host((size_t)std::max<int64_t>(c.used, 1));
  if (c.used > 0) CK(cudaMemcpy(host.data(), c.arena, (size_t)c.used * 16, cudaMemcpyDeviceToHost));
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(ctx, NEGF_B200_ERR_BAD_ARG, std::string("cannot write ") + path);
  // one entry per (lead, energy, broadening, tolerance): devices sharing a lead share it
  std::vector<std::pair<SgfFileEntry, int64_t>> out;
  std::unordered_map<uint64_t, int> seen;
  for (const auto& kv : c.map) {
    const DeviceRec& r = ctx->devs[kv.first.dev];
    SgfFileEntry e{r.lead_hash[kv.first.cont], r.desc.L[kv.first.cont], kv.first.maxit, kv.first.e, kv.first.eta,
                   kv.first.tol};
    const uint64_t k = fnv1a(fnv1a(fnv1a(e.hash, &e.e, 8), &e.eta, 8), &e.tol, 8);
    if (seen.count(k)) continue;
    seen[k] = 1;
    out.push_back({e, kv.second});
  }
  const int64_t n = (int64_t)out.size();
  bool ok = std::fwrite(kSgfMagic, 1, 8, f) == 8 && std::fwrite(&n, 8, 1, f) == 1;
  for (const auto& e : out) {
    ok = ok && std::fwrite(&e.first, sizeof(SgfFileEntry), 1, f) == 1;
    ok = ok && std::fwrite(host.data() + e.second, 16, (size_t)e.first.L * e.first.L, f) ==
                   (size_t)e.first.L * e.first.L;
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return fail(ctx, NEGF_B200_ERR_BAD_ARG, std::string("write error on ") + path);
  if (entries) *entries = n;
  return NEGF_B200_OK;
}

int negf_b200_sgf_cache_load(negf_b200_ctx* ctx, const char* path, int64_t* entries) {
  if (!ctx || !path) return NEGF_B200_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  SgfCache& c = ctx->sgf;
  if (c.mode == 0 || !c.arena) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "enable the SGF cache before loading into it");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream));
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(ctx, NEGF_B200_ERR_BAD_ARG, std::string("cannot read ") + path);
  char magic[8];
  int64_t n = 0, loaded = 0;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kSgfMagic, 8) == 0 && std::fread(&n, 8, 1, f) == 1 &&
            n >= 0;
  std::vector<SgfFileEntry> ents;
  std::vector<std::vector<double2>> vals;
  for (int64_t q = 0; ok && q < n; ++q) {
    SgfFileEntry e;
    ok = std::fread(&e, sizeof(e), 1, f) == 1 && e.L >= 1 && e.L <= negf::kMaxOrder;
    if (!ok) break;
    std::vector<double2> v((size_t)e.L * e.L);
    ok = std::fread(v.data(), 16, v.size(), f) == v.size();
    ents.push_back(e);
    vals.push_back(std::move(v));
  }
  std::fclose(f);
  if (!ok) return fail(ctx, NEGF_B200_ERR_BAD_ARG, std::string("not an SGF cache file or truncated: ") + path);
  for (size_t q = 0; q < ents.size(); ++q) {
    const SgfFileEntry& e = ents[q];
    const int64_t L2 = (int64_t)e.L * e.L;
    const std::vector<double2>& buf = vals[q];
    bool used_once = false;
    for (size_t d = 0; d < ctx->devs.size(); ++d) {
      const DeviceRec& r = ctx->devs[d];
      if (!r.live) continue;
      for (int k = 0; k < r.ncont; ++k) {
        if (r.lead_hash[k] != e.hash || r.desc.L[k] != e.L) continue;
        SgfKey key{(int32_t)d, k, e.e, e.eta, e.tol, e.maxit};
        if (c.map.count(key)) continue;
        if (c.used + L2 > c.cap) continue;                 // no room: computed when needed
        const int64_t off = c.used;
        CK(cudaMemcpy(c.arena + off, buf.data(), (size_t)L2 * 16, cudaMemcpyHostToDevice));
        c.used += (L2 + 15) & ~int64_t(15);
        c.map[key] = off;
        used_once = true;
      }
    }
    loaded += used_once ? 1 : 0;
  }
  if (entries) *entries = loaded;
  return NEGF_B200_OK;
}

int negf_b200_sgf_cache_stats(const negf_b200_ctx* ctx, int64_t* hits, int64_t* misses, int64_t* entries,
                              size_t* bytes_used) {
  if (!ctx) return NEGF_B200_ERR_BAD_ARG;
  if (hits) *hits = ctx->sgf.hits;
  if (misses) *misses = ctx->sgf.misses;
  if (entries) *entries = (int64_t)ctx->sgf.map.size();
  if (bytes_used) *bytes_used = (size_t)ctx->sgf.used * sizeof(double2);
  return NEGF_B200_OK;
}

// ---- host-buffer solves ----------------------------------------------------
static int check_pair(negf_b200_ctx* ctx, int npts, const int32_t* ids, int ni, int nf) {
  for (int p = 0; p < npts; ++p) {
    const DeviceRec& r = ctx->devs[ids[p]];
    if (ni < 1 || nf < 1 || ni > r.ncont || nf > r.ncont || (r.ncont > 1 && ni == nf))
      return fail(ctx, NEGF_B200_ERR_BAD_ARG, "contact pair (ni, nf) outside 1..ncont");
  }
  return NEGF_B200_OK;
}

static int check_pairs(negf_b200_ctx* ctx, int npts, const int32_t* ids, int npairs, const int32_t* ni,
                       const int32_t* nf) {
  for (int q = 0; q < npairs; ++q) {
    int st = check_pair(ctx, npts, ids, ni[q], nf[q]);
    if (st) return st;
  }
  return NEGF_B200_OK;
}

// The lock-step forms of 2-contact transmission solves (negf::mixed_run):
// the mixed-precision form (options.precision != 0: int8 tensor-core
// products) and the small-order FP64 form (precision 0, n <= 32, by
// options.schedule).  Both need one shape for every point of a call.
static int mixed_slices(const negf_b200_ctx* ctx) { return ctx->opt.precision == 1 ? 8 : ctx->opt.precision; }

struct LockShape {
  int n = 0, nbl = 0, left = -1, right = -1;
};

// Whether the points (host ids; null: every device the context holds) fit
// the lock-step forms: 2 contacts on blocks 1 and nbl in the same order, one
// PL size n for all layers and both leads, the same nbl, no tun_proj, no
// bound surface layers.  The reason in *why when not.
static bool lockstep_shape(negf_b200_ctx* ctx, int32_t npts, const int32_t* h_ids, LockShape* sh, std::string* why,
                           bool* bad_id) {
  *bad_id = false;
  std::vector<int> used;
  if (h_ids) {
    std::vector<char> seen(ctx->devs.size(), 0);
    for (int p = 0; p < npts; ++p) {
      if (h_ids[p] < 0 || h_ids[p] >= (int)ctx->devs.size() || !ctx->devs[h_ids[p]].live) {
        *bad_id = true;
        *why = "unknown device id";
        return false;
      }
      if (!seen[h_ids[p]]) { seen[h_ids[p]] = 1; used.push_back(h_ids[p]); }
    }
  } else {
    for (int i = 0; i < (int)ctx->devs.size(); ++i)
      if (ctx->devs[i].live) used.push_back(i);
  }
  if (used.empty()) { *why = "a device"; return false; }
  const DeviceRec& r0 = ctx->devs[used[0]];
  const int n = r0.nmax, nbl = r0.nbl;
  int left = -1, right = -1;
  for (int id : used) {
    const DeviceRec& r = ctx->devs[id];
    if (r.ncont != 2 || r.nbl < 2 || r.nbl != nbl || r.nmax != n || r.norb != nbl * n) {
      *why = "2 contacts and one PL size n for all layers of every point's device";
      return false;
    }
    int l = -1, rr = -1;
    for (int c = 0; c < 2; ++c) {
      if (r.desc.L[c] != n) { *why = "lead PL size = n"; return false; }
      if (r.cblk[c] == 1) l = c;
      if (r.cblk[c] == nbl) rr = c;
    }
    if (l < 0 || rr < 0 || l == rr) { *why = "the contacts on blocks 1 and nbl"; return false; }
    if (left >= 0 && (l != left || rr != right)) { *why = "the same contact order on every device"; return false; }
    if (r.desc.tun_mask) { *why = "no tun_proj"; return false; }
    if (r.desc.surf[0] > 0 || r.desc.surf[1] > 0) { *why = "no bound surface layers"; return false; }
    left = l; right = rr;
  }
  sh->n = n; sh->nbl = nbl; sh->left = left; sh->right = right;
  return true;
}

// Decides how a 2-contact transmission call runs: returns true when a
// lock-step form takes it (*slices = the int8 digits, 0 = the small-order
// FP64 form) or when the call must fail (*st set); false for the engine.
static bool lockstep_choice(negf_b200_ctx* ctx, int32_t npts, const int32_t* h_ids, bool single_pair, LockShape* sh,
                            int* slices, int* st, cudaStream_t stream) {
  *st = NEGF_B200_OK;
  const bool mixed = ctx->opt.precision != 0;
  if (!mixed && ctx->opt.schedule == 1) return false;
  const bool forced = mixed || ctx->opt.schedule == 2;
  const char* form = mixed ? "the mixed form (precision != 0)" : "lock step (schedule 2)";
  // lock step reads the decimation's active count back to the host, which a
  // stream capture cannot hold: the engine takes captured calls
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) {
    cudaGetLastError();
    cap = cudaStreamCaptureStatusNone;
  }
  if (cap != cudaStreamCaptureStatusNone) {
    if (!forced) return false;
    *st = fail(ctx, NEGF_B200_ERR_BAD_ARG, std::string(form) + " cannot run under stream capture");
    return true;
  }
  // the mixed form neither reads nor fills the SGF cache, so a context that keeps
  // one (a serving lane) runs it too; the FP64 lock step leaves such calls to the
  // engine, which uses the cache
  if (!single_pair || (ctx->sgf.mode && !mixed)) {
    if (!forced) return false;
    *st = fail(ctx, NEGF_B200_ERR_BAD_ARG,
               std::string(form) + (mixed ? " covers single-pair transmission solves"
                                          : " covers single-pair transmission solves without the SGF cache"));
    return true;
  }
  std::string why;
  bool bad_id = false;
  bool ok = lockstep_shape(ctx, npts, h_ids, sh, &why, &bad_id);
  if (ok && !mixed && sh->n > negf::kSmallMax) {
    ok = false;
    why = "orders n <= 32";
  }
  if (!ok && (forced || bad_id)) {
    *st = fail(ctx, NEGF_B200_ERR_BAD_ARG, bad_id ? why : std::string(form) + " needs " + why);
    return true;
  }
  if (!ok) return false;
  *slices = mixed ? mixed_slices(ctx) : 0;
  return true;
}

// The solves that only the engine runs (DOS, N-contact pairs, SCBA, the
// density matrix) refuse the options that ask for a lock-step form.
static int engine_only(negf_b200_ctx* ctx, const char* what) {
  if (ctx->opt.precision != 0)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG,
                std::string("the mixed form (precision != 0) covers single-pair transmission solves, not ") + what);
  if (ctx->opt.schedule == 2)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG,
                std::string("lock step (schedule 2) covers single-pair transmission solves, not ") + what);
  return NEGF_B200_OK;
}

// Runs a lock-step form on device arrays of ids and energies// Runs a lock-step form on device arrays of ids and energies: sizes the batch
// to the workspace and calls negf::mixed_run.
static int run_lockstep(negf_b200_ctx* ctx, int32_t npts, const int32_t* d_ids, const double* d_E, double eta,
                        double* d_T, int32_t* d_ncyc, int32_t* d_status, cudaStream_t s, const LockShape& sh,
                        int slices) {
  int st = sync_descs(ctx);
  if (st) return st;
  const int n = sh.n;
  // the mixed form: two full waves of the inversion (one CTA per matrix, two
  // per SM: 592 on a B200); the small form: the whole call at once up to 8192
  int batch = std::min<int>(npts, slices ? 4 * std::max(ctx->sms, 1) : 8192);
  if (ctx->ws_limit) batch = std::min(batch, negf::mixed_batch_for(ctx->ws_limit, n, slices));
  if (batch < 1) return fail(ctx, NEGF_B200_ERR_ADMISSION, "the workspace limit is below one point of lock step");
  for (;;) {
    st = grow(ctx, &ctx->ws, &ctx->ws_bytes, negf::mixed_ws_bytes(batch, n, slices));
    if (st == NEGF_B200_OK) break;
    if (batch == 1) return st;
    batch = (batch + 1) / 2;
  }
  negf::MixedArgs a;
  a.npts = npts; a.d_ids = d_ids; a.d_E = d_E; a.eta = eta; a.d_descs = ctx->d_descs;
  a.n = n; a.nbl = sh.nbl; a.left = sh.left; a.right = sh.right;
  a.sgf_tol = ctx->opt.sgf_tol; a.sgf_max_iter = ctx->opt.sgf_max_iter; a.slices = slices;
  a.d_T = d_T; a.d_ncyc = d_ncyc; a.d_status = d_status;
  a.launches = &ctx->launches;
  std::string msg;
  st = negf::mixed_run(a, ctx->ws, batch, s, &msg);
  if (st) return fail(ctx, st, (slices ? "mixed form: " : "lock step: ") + msg);
  return NEGF_B200_OK;
}

static int solve_host(negf_b200_ctx* ctx, int mode, int32_t npts, const int32_t* ids, const double* E,
                      double eta, double dos_delta, int32_t ni, int32_t nf, double* T, double* dos, int32_t* ncyc,
                      int32_t* status, const double* frm, const double* coupling, double* curr, double* lcurr,
                      double* ldens, int32_t* scba_iter, double* scba_err, int32_t npairs = 1,
                      const int32_t* pni = nullptr, const int32_t* pnf = nullptr, double* ledos = nullptr) {
  if (!ctx) return NEGF_B200_ERR_BAD_ARG;
  if (npts < 0 || (npts > 0 && (!ids || !E))) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "bad point arrays");
  if (npts == 0) return NEGF_B200_OK;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  LaunchShape sh;
  int st = shape_of(ctx, npts, ids, sh);
  if (st) return st;
  int ncont_pts = 0, nbl_pts = 0, norb_pts = 0, nldos_pts = 0;
  for (int p = 0; p < npts; ++p) {
    const DeviceRec& r = ctx->devs[ids[p]];
    ncont_pts = std::max(ncont_pts, r.ncont);
    nbl_pts = std::max(nbl_pts, r.nbl);
    norb_pts = std::max(norb_pts, r.norb);
    nldos_pts = std::max(nldos_pts, r.nldos);
  }
  if (npairs < 1 || (npairs > 1 && (!pni || !pnf)))
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "npairs must be >= 1 with ni/nf arrays");
  if (ledos && mode != negf::MODE_DOS) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "ledos needs the DOS solve");
  if (mode != negf::MODE_GN) {
    st = (npairs > 1) ? check_pairs(ctx, npts, ids, npairs, pni, pnf) : check_pair(ctx, npts, ids, ni, nf);
    if (st) return st;
  } else {
    for (int p = 0; p < npts; ++p)
      if (ctx->devs[ids[p]].nbl < 2) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "the Gn solve needs nbl >= 2");
    if (!frm) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "frm is required");
  }
  // staging
  size_t need = 0;
  {
    Carve c{nullptr};
    c.take<int32_t>(npts); c.take<double>(npts); c.take<double>((size_t)npts * npairs); c.take<int32_t>(npts);
    c.take<int32_t>(npts);
    if (dos || ledos) c.take<double>((size_t)npts * norb_pts);
    if (ledos) c.take<double>((size_t)npts * std::max(1, nldos_pts));
    if (npairs > 1) { c.take<int32_t>(npairs); c.take<int32_t>(npairs); }
    if (ctx->sgf.mode) { c.take<int64_t>((size_t)npts * sh.ncont_max); c.take<int64_t>((size_t)npts * sh.ncont_max); }
    if (frm) c.take<double>((size_t)npts * ncont_pts);
    if (coupling) c.take<double>((size_t)norb_pts);
    if (curr) c.take<double>((size_t)npts * ncont_pts);
    if (lcurr) c.take<double>((size_t)npts * std::max(1, nbl_pts - 1));
    if (ldens) c.take<double>((size_t)npts * nbl_pts);
    c.take<int32_t>(npts); c.take<double>(npts);
    need = c.off + 256;
  }
  st = grow(ctx, &ctx->io, &ctx->io_bytes, need);
  if (st) return st;
  Carve c{reinterpret_cast<char*>(ctx->io)};
  int32_t* d_ids = c.take<int32_t>(npts);
  double* d_E = c.take<double>(npts);
  double* d_T = c.take<double>((size_t)npts * npairs);
  int32_t* d_ncyc = c.take<int32_t>(npts);
  int32_t* d_st = c.take<int32_t>(npts);
  double* d_dos = (dos || ledos) ? c.take<double>((size_t)npts * norb_pts) : nullptr;
  double* d_ldos = ledos ? c.take<double>((size_t)npts * std::max(1, nldos_pts)) : nullptr;
  int32_t* d_pni = (npairs > 1) ? c.take<int32_t>(npairs) : nullptr;
  int32_t* d_pnf = (npairs > 1) ? c.take<int32_t>(npairs) : nullptr;
  // indexed by point * ncont_max of the launch (run_device sets a.ncont_max = sh.ncont_max)
  int64_t* d_sgf_in = ctx->sgf.mode ? c.take<int64_t>((size_t)npts * sh.ncont_max) : nullptr;
  int64_t* d_sgf_out = ctx->sgf.mode ? c.take<int64_t>((size_t)npts * sh.ncont_max) : nullptr;
  double* d_frm = frm ? c.take<double>((size_t)npts * ncont_pts) : nullptr;
  double* d_cpl = coupling ? c.take<double>((size_t)norb_pts) : nullptr;
  double* d_curr = curr ? c.take<double>((size_t)npts * ncont_pts) : nullptr;
  double* d_lcurr = lcurr ? c.take<double>((size_t)npts * std::max(1, nbl_pts - 1)) : nullptr;
  double* d_ldens = ldens ? c.take<double>((size_t)npts * nbl_pts) : nullptr;
  int32_t* d_it = c.take<int32_t>(npts);
  double* d_err = c.take<double>(npts);
  cudaStream_t s = ctx->stream;
  CK(cudaMemcpyAsync(d_ids, ids, npts * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_E, E, npts * 8, cudaMemcpyHostToDevice, s));
  if (d_frm) CK(cudaMemcpyAsync(d_frm, frm, (size_t)npts * ncont_pts * 8, cudaMemcpyHostToDevice, s));
  if (d_cpl) CK(cudaMemcpyAsync(d_cpl, coupling, (size_t)norb_pts * 8, cudaMemcpyHostToDevice, s));
  if (d_pni) CK(cudaMemcpyAsync(d_pni, pni, (size_t)npairs * 4, cudaMemcpyHostToDevice, s));
  if (d_pnf) CK(cudaMemcpyAsync(d_pnf, pnf, (size_t)npairs * 4, cudaMemcpyHostToDevice, s));
  LockShape lsh;
  int lslices = 0;
  if (mode != negf::MODE_T) {
    st = engine_only(ctx, "this solve");
    if (st) return st;
  }
  const bool lock = mode == negf::MODE_T && lockstep_choice(ctx, npts, ids, npairs == 1, &lsh, &lslices, &st, s);
  if (lock && st) return st;
  // the cache plan (which points read a cached gs, which fill a slot) only for
  // the engine: a lock-step form would leave the planned slots unfilled
  std::vector<int64_t> sgf_in, sgf_out;
  if (ctx->sgf.mode && !lock) {
    plan_sgf(ctx, npts, ids, E, eta, sh.ncont_max, sgf_in, sgf_out);
    CK(cudaMemcpyAsync(d_sgf_in, sgf_in.data(), sgf_in.size() * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_sgf_out, sgf_out.data(), sgf_out.size() * 8, cudaMemcpyHostToDevice, s));
  }
  if (lock) {
    st = run_lockstep(ctx, npts, d_ids, d_E, eta, d_T, d_ncyc, d_st, s, lsh, lslices);
    if (st) return st;
    std::vector<int32_t> hst(npts);
    if (T) CK(cudaMemcpyAsync(T, d_T, (size_t)npts * 8, cudaMemcpyDeviceToHost, s));
    if (ncyc) CK(cudaMemcpyAsync(ncyc, d_ncyc, npts * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hst.data(), d_st, npts * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (status) std::memcpy(status, hst.data(), npts * 4);
    return first_status(hst.data(), npts);
  }
  negf::EngineArgs a = base_args(ctx, mode, npts);
  a.dev_id = d_ids; a.energy = d_E; a.eta = eta; a.dos_delta = dos_delta; a.ni = ni; a.nf = nf;
  a.T = d_T; a.ncyc = d_ncyc; a.status = d_st;
  a.npairs = npairs; a.pair_ni = d_pni; a.pair_nf = d_pnf;
  a.dos = d_dos; a.dos_stride = norb_pts;
  a.ldos = d_ldos; a.ldos_stride = std::max(1, nldos_pts);
  a.sgf_in = d_sgf_in; a.sgf_out = d_sgf_out; a.sgf_arena = ctx->sgf.arena;
  a.frm = d_frm; a.frm_stride = ncont_pts; a.coupling = d_cpl;
  a.curr = d_curr; a.curr_stride = ncont_pts;
  a.lcurr = d_lcurr; a.lcurr_stride = std::max(1, nbl_pts - 1);
  a.ldens = d_ldens; a.ldens_stride = nbl_pts;
  a.scba_iter = d_it; a.scba_err = d_err;
  st = run_device(ctx, a, sh, s);
  if (st) return st;
  std::vector<int32_t> hst(npts);
  const size_t b_T = T ? (size_t)npts * npairs * 8 : 0;
  const size_t b_ledos = (ledos && nldos_pts > 0) ? (size_t)npts * nldos_pts * 8 : 0;
  const size_t b_dos = dos ? (size_t)npts * norb_pts * 8 : 0;
  const size_t b_curr = curr ? (size_t)npts * ncont_pts * 8 : 0;
  const size_t b_lcurr = lcurr ? (size_t)npts * std::max(1, nbl_pts - 1) * 8 : 0;
  const size_t b_ldens = ldens ? (size_t)npts * nbl_pts * 8 : 0;
  ReadBack rb(ctx, s, ReadBack::staged_size(b_T) + ReadBack::staged_size(b_ledos) + ReadBack::staged_size(b_dos) +
                          ReadBack::staged_size(b_curr) + ReadBack::staged_size(b_lcurr) +
                          ReadBack::staged_size(b_ldens));
  CK(rb.copy(T, d_T, b_T));
  CK(rb.copy(ledos, d_ldos, b_ledos));
  if (ncyc) CK(cudaMemcpyAsync(ncyc, d_ncyc, npts * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(hst.data(), d_st, npts * 4, cudaMemcpyDeviceToHost, s));
  CK(rb.copy(dos, d_dos, b_dos));
  CK(rb.copy(curr, d_curr, b_curr));
  CK(rb.copy(lcurr, d_lcurr, b_lcurr));
  CK(rb.copy(ldens, d_ldens, b_ldens));
  if (scba_iter) CK(cudaMemcpyAsync(scba_iter, d_it, npts * 4, cudaMemcpyDeviceToHost, s));
  if (scba_err) CK(cudaMemcpyAsync(scba_err, d_err, npts * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  rb.finish();
  if (status) std::memcpy(status, hst.data(), npts * 4);
  return first_status(hst.data(), npts);
}

int negf_b200_transmission(negf_b200_ctx* ctx, int32_t npts, const int32_t* device_id, const double* energy,
                           double eta, int32_t ni, int32_t nf, double* T, int32_t* ncyc, int32_t* status) {
  return solve_host(ctx, negf::MODE_T, npts, device_id, energy, eta, 0.0, ni, nf, T, nullptr, ncyc, status,
                    nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
}

int negf_b200_transmission_dos(negf_b200_ctx* ctx, int32_t npts, const int32_t* device_id, const double* energy,
                               double eta, double dos_delta, int32_t ni, int32_t nf, double* T, double* dos,
                               int32_t* ncyc, int32_t* status) {
  return solve_host(ctx, negf::MODE_DOS, npts, device_id, energy, eta, dos_delta, ni, nf, T, dos, ncyc, status,
                    nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
}

int negf_b200_meir_wingreen(negf_b200_ctx* ctx, int32_t npts, const int32_t* device_id, const double* energy,
                            double eta, const double* frm, const double* coupling, double* curr,
                            double* layer_curr, double* layer_dens, int32_t* scba_iter, double* scba_err,
                            int32_t* ncyc, int32_t* status) {
  return solve_host(ctx, negf::MODE_GN, npts, device_id, energy, eta, 0.0, 1, 2, nullptr, nullptr, ncyc, status,
                    frm, coupling, curr, layer_curr, layer_dens, scba_iter, scba_err);
}

int negf_b200_transmissions(negf_b200_ctx* ctx, int32_t npts, const int32_t* device_id, const double* energy,
                            double eta, double dos_delta, int32_t npairs, const int32_t* ni, const int32_t* nf,
                            double* T, double* ledos, int32_t* ncyc, int32_t* status) {
  if (!ctx || npairs < 1 || !ni || !nf) return NEGF_B200_ERR_BAD_ARG;
  return solve_host(ctx, ledos ? negf::MODE_DOS : negf::MODE_T, npts, device_id, energy, eta, ledos ? dos_delta : 0.0,
                    ni[0], nf[0], T, nullptr, ncyc, status, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                    nullptr, npairs, ni, nf, ledos);
}

namespace {

// Sum of w_p * (Gr or Gn blocks) over the points of one device (engine MODE_RHO
// or MODE_GN with block accumulation), copied back to T (diag | upper | lower).
int accumulate_blocks(negf_b200_ctx* ctx, int mode, int32_t device_id, int32_t npts, const double* e_re,
                      const double* e_im, double eta, const double* weight, const double* frm,
                      const double* coupling, std::vector<double2>& T, std::vector<int>& pl, int64_t& nd,
                      int64_t& no, int32_t* ncyc, int32_t* status, std::vector<double2>* outer = nullptr,
                      int64_t* nm_out = nullptr) {
  if (int e = engine_only(ctx, "the density matrix")) return e;
  if (device_id < 0 || device_id >= (int)ctx->devs.size() || !ctx->devs[device_id].live)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "unknown device id");
  const DeviceRec& r = ctx->devs[device_id];
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  pl.assign(r.nbl, 0);
  CK(cudaMemcpy(pl.data(), r.desc.pl, r.nbl * 4, cudaMemcpyDeviceToHost));
  nd = no = 0;
  for (int i = 0; i < r.nbl; ++i) {
    nd += (int64_t)pl[i] * pl[i];
    if (i + 1 < r.nbl) no += (int64_t)pl[i] * pl[i + 1];
  }
  T.assign((size_t)(nd + 2 * no), make_double2(0.0, 0.0));
  int64_t nm = 0;   // outer blocks: sum over contacts of n_cb x L (the hmc layout)
  for (int c = 0; c < r.ncont; ++c) nm += (int64_t)pl[r.desc.cblk[c] - 1] * r.desc.L[c];
  if (nm_out) *nm_out = nm;
  if (outer) outer->assign((size_t)(2 * nm), make_double2(0.0, 0.0));
  if (outer)
    for (int c = 0; c < r.ncont; ++c)
      if (r.desc.surf[c] > 0)
        return fail(ctx, NEGF_B200_ERR_BAD_ARG, "outer blocks of a contact with bound surface layers are not built");
  if (npts == 0) return NEGF_B200_OK;
  if (mode == negf::MODE_GN && r.nbl < 2) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "the Gn solve needs nbl >= 2");
  std::vector<int32_t> ids(npts, device_id);
  LaunchShape sh;
  int st = shape_of(ctx, npts, ids.data(), sh);
  if (st) return st;
  size_t need = 0;
  {
    Carve c{nullptr};
    c.take<int32_t>(npts); c.take<double>(npts); c.take<double>(npts); c.take<double2>(npts);
    c.take<int32_t>(npts); c.take<int32_t>(npts); c.take<double2>((size_t)(nd + 2 * no));
    c.take<double>((size_t)npts * r.ncont); c.take<double>((size_t)r.norb); c.take<int32_t>(npts);
    c.take<double>(npts);
    if (outer) c.take<double2>((size_t)(2 * nm));
    need = c.off + 256;
  }
  st = grow(ctx, &ctx->io, &ctx->io_bytes, need);
  if (st) return st;
  Carve c{reinterpret_cast<char*>(ctx->io)};
  int32_t* d_ids = c.take<int32_t>(npts);
  double* d_re = c.take<double>(npts);
  double* d_im = c.take<double>(npts);
  double2* d_w = c.take<double2>(npts);
  int32_t* d_nc = c.take<int32_t>(npts);
  int32_t* d_st = c.take<int32_t>(npts);
  double2* d_acc = c.take<double2>((size_t)(nd + 2 * no));
  double* d_frm = c.take<double>((size_t)npts * r.ncont);
  double* d_cpl = c.take<double>((size_t)r.norb);
  int32_t* d_it = c.take<int32_t>(npts);
  double* d_err = c.take<double>(npts);
  double2* d_outer = outer ? c.take<double2>((size_t)(2 * nm)) : nullptr;
  cudaStream_t s = ctx->stream;
  if (d_outer) CK(cudaMemsetAsync(d_outer, 0, (size_t)(2 * nm) * 16, s));
  CK(cudaMemcpyAsync(d_ids, ids.data(), npts * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_re, e_re, npts * 8, cudaMemcpyHostToDevice, s));
  if (e_im) CK(cudaMemcpyAsync(d_im, e_im, npts * 8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_w, weight, npts * 16, cudaMemcpyHostToDevice, s));
  if (frm) CK(cudaMemcpyAsync(d_frm, frm, (size_t)npts * r.ncont * 8, cudaMemcpyHostToDevice, s));
  if (coupling) CK(cudaMemcpyAsync(d_cpl, coupling, (size_t)r.norb * 8, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(d_acc, 0, (size_t)(nd + 2 * no) * 16, s));
  negf::EngineArgs a = base_args(ctx, mode, npts);
  a.dev_id = d_ids; a.energy = d_re; a.energy_im = d_im; a.weight = d_w; a.eta = eta;
  a.acc_d = d_acc; a.acc_u = d_acc + nd; a.acc_l = d_acc + nd + no;
  a.acc_lc = d_outer; a.acc_cl = d_outer ? d_outer + nm : nullptr;
  a.ncyc = d_nc; a.status = d_st;
  if (mode == negf::MODE_GN) {
    a.frm = d_frm; a.frm_stride = r.ncont; a.coupling = coupling ? d_cpl : nullptr;
    a.scba_iter = d_it; a.scba_err = d_err;
  }
  st = run_device(ctx, a, sh, s);
  if (st) return st;
  std::vector<int32_t> hst(npts);
  CK(cudaMemcpyAsync(T.data(), d_acc, T.size() * 16, cudaMemcpyDeviceToHost, s));
  if (d_outer) CK(cudaMemcpyAsync(outer->data(), d_outer, outer->size() * 16, cudaMemcpyDeviceToHost, s));
  if (ncyc) CK(cudaMemcpyAsync(ncyc, d_nc, npts * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(hst.data(), d_st, npts * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (status) std::memcpy(status, hst.data(), npts * 4);
  st = first_status(hst.data(), npts);
  if (st && st != NEGF_B200_ERR_NOT_CONVERGED && st != NEGF_B200_ERR_SCBA_NOT_CONVERGED) return st;
  return NEGF_B200_OK;
}

void store_blocks(const double2* src, int64_t n, double* dst) {
  if (dst) std::memcpy(dst, src, (size_t)n * 16);
}

}  // namespace

int negf_b200_density(negf_b200_ctx* ctx, int32_t device_id, int32_t npts, const double* e_re, const double* e_im,
                      const double* weight, double* rho_diag, double* rho_upper, double* rho_lower, double* rho_dc,
                      double* rho_cd, int32_t* ncyc, int32_t* status) {
  if (!ctx) return NEGF_B200_ERR_BAD_ARG;
  if (npts < 0 || (npts > 0 && (!e_re || !e_im || !weight))) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "bad point arrays");
  std::lock_guard<std::mutex> lk(ctx->mu);
  std::vector<double2> T, Tout;
  std::vector<int> pl;
  int64_t nd = 0, no = 0, nm = 0;
  const bool want_outer = rho_dc || rho_cd;
  int st = accumulate_blocks(ctx, negf::MODE_RHO, device_id, npts, e_re, e_im, 0.0, weight, nullptr, nullptr, T, pl,
                             nd, no, ncyc, status, want_outer ? &Tout : nullptr, &nm);
  if (st) return st;
  if (want_outer) {
    // calculate_Gr_outer keeps the entries on the pattern of Tlc = E SMC - HMC (and of
    // Tcl for the lower block): the nonzeros of HMC or SMC; then zspectral pairs them
    const DeviceRec& r = ctx->devs[device_id];
    std::vector<double2> hmc((size_t)std::max<int64_t>(nm, 1)), smc;
    CK(cudaMemcpy(hmc.data(), r.desc.hmc, (size_t)nm * 16, cudaMemcpyDeviceToHost));
    if (r.desc.smc) {
      smc.resize((size_t)nm);
      CK(cudaMemcpy(smc.data(), r.desc.smc, (size_t)nm * 16, cudaMemcpyDeviceToHost));
    }
    auto nz = [&](int64_t q) {
      return hmc[q].x != 0.0 || hmc[q].y != 0.0 || (!smc.empty() && (smc[q].x != 0.0 || smc[q].y != 0.0));
    };
    const double2* Tlc = Tout.data();
    const double2* Tcl = Tlc + nm;
    int64_t om = 0;
    for (int c = 0; c < r.ncont; ++c) {
      const int n = pl[r.desc.cblk[c] - 1], L = r.desc.L[c];
      for (int j = 0; j < L; ++j)
        for (int q = 0; q < n; ++q) {
          const int64_t idc = om + q + (int64_t)j * n;   // (q, j) of the n x L block
          const int64_t icd = om + j + (int64_t)q * L;   // (j, q) of the L x n block
          const bool on = nz(idc);
          const double2 lc = on ? Tlc[idc] : make_double2(0.0, 0.0);
          const double2 cl = on ? Tcl[icd] : make_double2(0.0, 0.0);
          if (rho_dc) { rho_dc[2 * idc] = -(lc.y + cl.y); rho_dc[2 * idc + 1] = lc.x - cl.x; }   // i (lc - conj(cl))
          if (rho_cd) { rho_cd[2 * icd] = -(cl.y + lc.y); rho_cd[2 * icd + 1] = cl.x - lc.x; }   // i (cl - conj(lc))
        }
      om += (int64_t)n * L;
    }
  }
  const int nbl = (int)pl.size();
  // rho = i (T - T^dag) over the tridiagonal blocks (zspectral, src/integrations.F90:893)
  const double2* Td = T.data();
  const double2* Tu = Td + nd;
  const double2* Tl = Tu + no;
  auto ispec = [](double2 x, double2 y) {   // i (x - conj(y))
    return make_double2(-(x.y + y.y), x.x - y.x);
  };
  int64_t od = 0, oo = 0;
  for (int i = 0; i < nbl; ++i) {
    const int n = pl[i];
    if (rho_diag)
      for (int c = 0; c < n; ++c)
        for (int q = 0; q < n; ++q) {
          const double2 v = ispec(Td[od + q + (int64_t)c * n], Td[od + c + (int64_t)q * n]);
          rho_diag[2 * (od + q + (int64_t)c * n)] = v.x;
          rho_diag[2 * (od + q + (int64_t)c * n) + 1] = v.y;
        }
    if (i + 1 < nbl) {
      const int m = pl[i + 1];   // upper block n x m, lower block m x n
      for (int c = 0; c < m; ++c)
        for (int q = 0; q < n; ++q) {
          const double2 v = ispec(Tu[oo + q + (int64_t)c * n], Tl[oo + c + (int64_t)q * m]);
          if (rho_upper) { rho_upper[2 * (oo + q + (int64_t)c * n)] = v.x; rho_upper[2 * (oo + q + (int64_t)c * n) + 1] = v.y; }
        }
      for (int c = 0; c < n; ++c)
        for (int q = 0; q < m; ++q) {
          const double2 v = ispec(Tl[oo + q + (int64_t)c * m], Tu[oo + c + (int64_t)q * n]);
          if (rho_lower) { rho_lower[2 * (oo + q + (int64_t)c * m)] = v.x; rho_lower[2 * (oo + q + (int64_t)c * m) + 1] = v.y; }
        }
      oo += (int64_t)n * m;
    }
    od += (int64_t)n * n;
  }
  return NEGF_B200_OK;
}

int negf_b200_density_neq(negf_b200_ctx* ctx, int32_t device_id, int32_t npts, const double* energy, double eta,
                          const double* weight, const double* frm, const double* coupling, double* rho_diag,
                          double* rho_upper, double* rho_lower, double* rho_dc, double* rho_cd, int32_t* ncyc,
                          int32_t* status) {
  if (!ctx) return NEGF_B200_ERR_BAD_ARG;
  if (npts < 0 || (npts > 0 && (!energy || !weight || !frm))) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "bad point arrays");
  std::lock_guard<std::mutex> lk(ctx->mu);
  std::vector<double2> T, Tout;
  std::vector<int> pl;
  int64_t nd = 0, no = 0, nm = 0;
  const bool want_outer = rho_dc || rho_cd;
  int st = accumulate_blocks(ctx, negf::MODE_GN, device_id, npts, energy, nullptr, eta, weight, frm, coupling, T, pl,
                             nd, no, ncyc, status, want_outer ? &Tout : nullptr, &nm);
  if (st) return st;
  if (want_outer) {
    // calculate_Gn_outer masks Gn(cb,c) with Tlc's pattern (the nonzeros of HMC or SMC) and
    // takes Gn(c,cb) as the dagger of the masked block; the sums are masked the same way
    const DeviceRec& r = ctx->devs[device_id];
    std::vector<double2> hmc((size_t)std::max<int64_t>(nm, 1)), smc;
    CK(cudaMemcpy(hmc.data(), r.desc.hmc, (size_t)nm * 16, cudaMemcpyDeviceToHost));
    if (r.desc.smc) {
      smc.resize((size_t)nm);
      CK(cudaMemcpy(smc.data(), r.desc.smc, (size_t)nm * 16, cudaMemcpyDeviceToHost));
    }
    int64_t om = 0;
    for (int c = 0; c < r.ncont; ++c) {
      const int n = pl[r.desc.cblk[c] - 1], L = r.desc.L[c];
      for (int j = 0; j < L; ++j)
        for (int q = 0; q < n; ++q) {
          const int64_t idc = om + q + (int64_t)j * n;   // (q, j) of the n x L block
          const int64_t icd = om + j + (int64_t)q * L;   // (j, q) of the L x n block
          const bool on = hmc[idc].x != 0.0 || hmc[idc].y != 0.0 ||
                          (!smc.empty() && (smc[idc].x != 0.0 || smc[idc].y != 0.0));
          const double2 lc = on ? Tout[idc] : make_double2(0.0, 0.0);
          const double2 cl = on ? Tout[nm + icd] : make_double2(0.0, 0.0);
          if (rho_dc) { rho_dc[2 * idc] = lc.x; rho_dc[2 * idc + 1] = lc.y; }
          if (rho_cd) { rho_cd[2 * icd] = cl.x; rho_cd[2 * icd + 1] = cl.y; }
        }
      om += (int64_t)n * L;
    }
  }
  // real_axis_int adds the sum itself to rho (no spectral combination, :1166-1170)
  store_blocks(T.data(), nd, rho_diag);
  store_blocks(T.data() + nd, no, rho_upper);
  store_blocks(T.data() + nd + no, no, rho_lower);
  return NEGF_B200_OK;
}

// ---- device-pointer solve (inputs already resident in HBM) ------------------
int negf_b200_transmission_dev(negf_b200_ctx* ctx, int32_t npts, const int32_t* d_device_id,
                               const double* d_energy, double eta, int32_t ni, int32_t nf, double* d_T,
                               int32_t* d_ncyc, int32_t* d_status, void* stream) {
  if (!ctx || npts < 0) return NEGF_B200_ERR_BAD_ARG;
  if (npts == 0) return NEGF_B200_OK;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  {
    LockShape lsh;
    int lslices = 0, lst = 0;
    const cudaStream_t ls = stream ? (cudaStream_t)stream : ctx->stream;
    if (lockstep_choice(ctx, npts, nullptr, true, &lsh, &lslices, &lst, ls)) {
      if (lst) return lst;
      return run_lockstep(ctx, npts, d_device_id, d_energy, eta, d_T, d_ncyc, d_status, ls, lsh, lslices);
    }
  }
  LaunchShape sh;
  int st = shape_of(ctx, npts, nullptr, sh);
  if (st) return st;
  negf::EngineArgs a = base_args(ctx, negf::MODE_T, npts);
  a.dev_id = d_device_id; a.energy = d_energy; a.eta = eta; a.ni = ni; a.nf = nf;
  a.T = d_T; a.ncyc = d_ncyc; a.status = d_status;
  return run_device(ctx, a, sh, stream ? (cudaStream_t)stream : ctx->stream);
}

int negf_b200_transmission_dos_dev(negf_b200_ctx* ctx, int32_t npts, const int32_t* d_device_id,
                                   const double* d_energy, double eta, double dos_delta, int32_t ni, int32_t nf,
                                   double* d_T, double* d_dos, int64_t dos_stride, int32_t* d_ncyc,
                                   int32_t* d_status, void* stream) {
  if (!ctx || npts < 0) return NEGF_B200_ERR_BAD_ARG;
  if (npts == 0) return NEGF_B200_OK;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  int st = engine_only(ctx, "the DOS solve");
  if (st) return st;
  LaunchShape sh;
  st = shape_of(ctx, npts, nullptr, sh);
  if (st) return st;
  negf::EngineArgs a = base_args(ctx, negf::MODE_DOS, npts);
  a.dev_id = d_device_id; a.energy = d_energy; a.eta = eta; a.dos_delta = dos_delta; a.ni = ni; a.nf = nf;
  a.T = d_T; a.dos = d_dos; a.dos_stride = dos_stride; a.ncyc = d_ncyc; a.status = d_status;
  return run_device(ctx, a, sh, stream ? (cudaStream_t)stream : ctx->stream);
}

int negf_b200_meir_wingreen_dev(negf_b200_ctx* ctx, int32_t npts, const int32_t* d_device_id,
                                const double* d_energy, double eta, const double* d_frm,
                                const double* d_coupling, double* d_curr, double* d_layer_curr,
                                double* d_layer_dens, int32_t* d_scba_iter, double* d_scba_err, int32_t* d_ncyc,
                                int32_t* d_status, int32_t cont_stride, int32_t layer_stride, void* stream) {
  if (!ctx || npts < 0) return NEGF_B200_ERR_BAD_ARG;
  if (npts == 0) return NEGF_B200_OK;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  if (!d_device_id || !d_energy || !d_frm || !d_scba_iter || !d_scba_err || !d_status)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "device_id, energy, frm, scba_iter, scba_err and status are required");
  if (int e = engine_only(ctx, "the SCBA solve")) return e;
  LaunchShape sh;
  int st = shape_of(ctx, npts, nullptr, sh);
  if (st) return st;
  for (const DeviceRec& r : ctx->devs)
    if (r.live && r.nbl < 2) return fail(ctx, NEGF_B200_ERR_BAD_ARG, "the Gn solve needs nbl >= 2 on every device");
  if (cont_stride < sh.ncont_max || layer_stride < sh.nbl_max)
    return fail(ctx, NEGF_B200_ERR_BAD_ARG, "cont_stride / layer_stride below the largest ncont / nbl");
  negf::EngineArgs a = base_args(ctx, negf::MODE_GN, npts);
  a.dev_id = d_device_id; a.energy = d_energy; a.eta = eta; a.ni = 1; a.nf = 2;
  a.ncyc = d_ncyc; a.status = d_status;
  a.frm = d_frm; a.frm_stride = cont_stride; a.coupling = d_coupling;
  a.curr = d_curr; a.curr_stride = cont_stride;
  a.lcurr = d_layer_curr; a.lcurr_stride = layer_stride;
  a.ldens = d_layer_dens; a.ldens_stride = layer_stride;
  a.scba_iter = d_scba_iter; a.scba_err = d_scba_err;
  return run_device(ctx, a, sh, stream ? (cudaStream_t)stream : ctx->stream);
}

// ---- tracing ----------------------------------------------------------------
int negf_b200_set_tracing(negf_b200_ctx* ctx, int32_t enable) {
  if (!ctx) return NEGF_B200_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  if (enable && !ctx->d_trace) {
    if (cudaMalloc(&ctx->d_trace, NEGF_B200_TRACE_NPHASE * sizeof(unsigned long long)) != cudaSuccess) {
      cudaGetLastError();
      ctx->d_trace = nullptr;
      return fail(ctx, NEGF_B200_ERR_NOMEM, "trace buffer");
    }
    CK(cudaMemset(ctx->d_trace, 0, NEGF_B200_TRACE_NPHASE * sizeof(unsigned long long)));
  }
  ctx->trace = enable != 0;
  return NEGF_B200_OK;
}

int negf_b200_get_trace(negf_b200_ctx* ctx, uint64_t* cycles) {
  if (!ctx || !cycles) return NEGF_B200_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  std::memset(cycles, 0, NEGF_B200_TRACE_NPHASE * sizeof(uint64_t));
  if (!ctx->d_trace) return NEGF_B200_OK;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, NEGF_B200_ERR_CUDA, "cudaSetDevice");
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(cycles, ctx->d_trace, NEGF_B200_TRACE_NPHASE * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  CK(cudaMemset(ctx->d_trace, 0, NEGF_B200_TRACE_NPHASE * sizeof(unsigned long long)));
  return NEGF_B200_OK;
}

// ---- primitives -------------------------------------------------------------
int negf_b200_zgemm_batched(int32_t batch, int32_t m, int32_t n, int32_t k, const double* alpha, const double* A,
                            int64_t strideA, const double* B, int64_t strideB, const double* beta, double* C,
                            int64_t strideC, int32_t dagger, void* stream) {
  if (batch < 0 || m < 0 || n < 0 || k < 0 || !alpha || !beta || (dagger < 0 || dagger > 2))
    return NEGF_B200_ERR_BAD_ARG;
  if (batch == 0 || m == 0 || n == 0) return NEGF_B200_OK;
  if (!A || !B || !C) return NEGF_B200_ERR_BAD_ARG;
  cudaError_t e = negf::launch_zgemm_batched(
      batch, m, n, k, make_double2(alpha[0], alpha[1]), (const double2*)A, strideA / 2, (const double2*)B,
      strideB / 2, make_double2(beta[0], beta[1]), (double2*)C, strideC / 2, dagger, (cudaStream_t)stream);
  return e == cudaSuccess ? NEGF_B200_OK : NEGF_B200_ERR_CUDA;
}

size_t negf_b200_zgemm_i8_work_bytes(int32_t batch, int32_t m, int32_t n, int32_t k, int32_t slices) {
  if (batch <= 0 || m <= 0 || n <= 0 || k <= 0 || slices < negf::kOzMinSlices || slices > negf::kOzMaxSlices)
    return 0;
  return negf::ozaki_layout(batch, m, n, k, slices).total + 256;
}

int negf_b200_zgemm_batched_i8(int32_t batch, int32_t m, int32_t n, int32_t k, const double* alpha,
                               const double* A, int64_t strideA, const double* B, int64_t strideB,
                               const double* beta, double* C, int64_t strideC, int32_t slices, void* work,
                               int32_t* status, void* stream) {
  if (batch < 0 || m < 0 || n < 0 || k < 0 || k > negf::kMaxOrder || batch > 65535 || !alpha || !beta ||
      slices < negf::kOzMinSlices || slices > negf::kOzMaxSlices)
    return NEGF_B200_ERR_BAD_ARG;
  if (batch == 0 || m == 0 || n == 0) return NEGF_B200_OK;
  if (!A || !B || !C || !work || k == 0) return NEGF_B200_ERR_BAD_ARG;
  // the workspace is used from its first 256-byte boundary
  uint8_t* w = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(work) + 255) & ~uintptr_t(255));
  cudaError_t e = negf::launch_ozaki_zgemm(batch, m, n, k, make_double2(alpha[0], alpha[1]), (const double2*)A,
                                           strideA / 2, (const double2*)B, strideB / 2,
                                           make_double2(beta[0], beta[1]), (double2*)C, strideC / 2, slices, w,
                                           nullptr, status, (cudaStream_t)stream);
  return e == cudaSuccess ? NEGF_B200_OK : NEGF_B200_ERR_CUDA;
}

size_t negf_b200_zinv_work_bytes(int32_t batch, int32_t n) {
  if (batch <= 0 || n <= 0) return 0;
  return (size_t)batch * negf::zinv_batched_work_elems(n) * 16 + 16;
}

int negf_b200_zinv_batched(int32_t batch, int32_t n, const double* A, double* Ainv, int32_t* info, void* work,
                           void* stream) {
  if (batch < 0 || n < 0 || n > negf::kMaxOrder) return NEGF_B200_ERR_BAD_ARG;
  if (batch == 0 || n == 0) return NEGF_B200_OK;
  // work may be null where the inversion needs no buffers of its own (n <= 64): the residual probe is skipped
  if (!A || !Ainv || (negf::zinv_batched_work_elems(n) > 2 * (size_t)n * n && !work)) return NEGF_B200_ERR_BAD_ARG;
  cudaError_t e = negf::launch_zinv_batched(batch, n, (const double2*)A, (double2*)Ainv, info, (double2*)work,
                                            (cudaStream_t)stream);
  return e == cudaSuccess ? NEGF_B200_OK : NEGF_B200_ERR_CUDA;
}

size_t negf_b200_decimation_work_bytes(int32_t batch, int32_t n) {
  if (batch <= 0 || n <= 0) return 0;
  return (size_t)batch * negf::decimation_batched_work_elems(n) * 16 + 16;
}

int negf_b200_decimation_batched(int32_t batch, int32_t n, const double* Ao, const double* Bo, const double* Co,
                                 double* Go, int32_t* ncyc, double tol, int32_t max_iter, void* work,
                                 void* stream) {
  if (batch < 0 || n < 0 || n > negf::kMaxOrder || tol <= 0.0 || max_iter < 1) return NEGF_B200_ERR_BAD_ARG;
  if (batch == 0 || n == 0) return NEGF_B200_OK;
  if (!Ao || !Bo || !Co || !Go || !work) return NEGF_B200_ERR_BAD_ARG;
  cudaError_t e = negf::launch_decimation_batched(batch, n, (const double2*)Ao, (const double2*)Bo,
                                                  (const double2*)Co, (double2*)Go, ncyc, tol, max_iter,
                                                  (double2*)work, (cudaStream_t)stream);
  return e == cudaSuccess ? NEGF_B200_OK : NEGF_B200_ERR_CUDA;
}

}  // extern "C"
