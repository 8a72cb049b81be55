// Batched FP32-compensated step: many independent grids (uneven shapes, each
// with its own dt, beam, materials and Ez capture) advanced together over
// one device work list (sm_100a).
//
// Upstream runs one SolverFIT3D.wakesolve per geometry (wakis/routines.py:
// 231-482); a batch of small grids launched one by one leaves most of the
// GPU idle in each launch's tail.  Here the work of a step is a list of
// items over all instances:
//
//   phase A  the TMA tiles of every instance (comp_tile, the block work of
//            the one-grid kernel, fit_tma_comp.cuh) and, for instances whose
//            z faces are not PEC-masked, the H rows of the four z-boundary
//            planes (comp_shell_h);
//   phase B  (only with such instances) the E rows of those planes, which
//            read the new H of the tiles next to them (comp_shell_e).
//
// Two launch forms run the lists:
//
// * persistent (WK_BATCH_PERSISTENT): ONE cooperative launch of (SMs x
//   blocks per SM) blocks for a chunk of steps.  Blocks claim items in order
//   (step, phase, item) from one atomic ticket.  Instances do not depend on
//   each other, so there is no grid-wide barrier: before an item of instance
//   q the block waits until q's own earlier work is done (phase-A items of
//   q's previous steps, and for a phase-B item those of this step), counted
//   by per-instance completion counters.  Every item a block waits for was
//   claimed before its own, by a block that is resident (cooperative
//   launch), so the waits always end; each is also bounded by a
//   %globaltimer deadline, after which the block records the failure in the
//   status word and all blocks leave.
// * phases (WK_BATCH_PHASES): per step, one launch per list (64x8 and 32x16
//   tiles whose compensation words come by TMA, the same with per-thread
//   loads, boundary-plane H rows, boundary-plane E rows); the stream orders
//   them.
//
// Each instance has its own tile shape (wk_fit_desc.tile_rows: 32x16 or
// 64x8 tiles), so that grids whose x extent lies just above a multiple of
// 64 do not leave most lanes of their last tile column idle.
//
// Each item reads its instance's parameters from the workspace; the TMA
// descriptors of every instance and buffer parity live there too.  The
// parity of the live buffers of step t is par_ref ^ ((t - t_ref) & 1), so a
// captured chunk can be replayed with a device step counter.
#include <cstring>
#include <vector>

#include "fit_tma_comp.cuh"

#include "abi_internal.h"

namespace wk {

namespace {

constexpr long long kDepNs = 2000000000LL;   // 2 s of %globaltimer per dependency wait
constexpr long long kDepPolls = 1LL << 28;

// Zeroed at the start of every run (with the completion counters after it).
struct BatchSync {
  unsigned ticket;          // next item (step, phase, index) to claim
  int abort;                // a block gave up: every block leaves
  int pad[2];
};

struct BatchInst {
  FitParams<double> p;
  CompState cs[2];          // the state with E[par] live, par = 0, 1
  long long t_ref;          // the step index whose step reads parity par_ref
  int par_ref;
  int ct;                   // compensation words by TMA (Nx % 8 == 0)
  unsigned nA, nB;          // items of this instance in phase A, phase B
  int tw;                   // tile width: 64 (64x8 tiles) or 32 (32x16)
};
static_assert(sizeof(FitParams<double>) % 8 == 0, "parameters are copied as 8-byte words");
static_assert(sizeof(CompState) % 8 == 0, "state pointers are copied as 8-byte words");

// kind 0: tile (a = bx | by << 16, b = bz | KC << 16); 1: H rows of the
// z-boundary plane a (0, 1, 2, 3 for k = 0, 1, Nz-2, Nz-1); 2: E rows of it
struct BatchItem {
  int inst, kind, a, b;
};

struct BatchArgs {
  BatchSync* sync;
  unsigned* done;           // [inst][phase] completed items of the run
  const BatchInst* insts;
  const CompMaps* maps;     // [inst][parity]
  const BatchItem* items[2];
  int n_items[2];
  int n_steps;
  long long step0;
  const long long* step_dev;
  long long wait_ns;        // bound of each dependency wait
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Wait (thread 0) until instance counters reach the given counts, the
// launch is aborted, or limit_ns passes; true when the counts were reached.
__device__ bool wait_done(const unsigned* done, unsigned needA, unsigned needB,
                          const int* abort, long long limit_ns) {
  if (ld_acquire_u32(reinterpret_cast<const unsigned*>(abort))) return false;
  if (ld_acquire_u32(done) >= needA && ld_acquire_u32(done + 1) >= needB) return true;
  const unsigned long long t0 = globaltimer_ns();
  for (long long it = 0; it < kDepPolls; it++) {
    __nanosleep(64);
    if (ld_acquire_u32(done) >= needA && ld_acquire_u32(done + 1) >= needB) return true;
    if (ld_acquire_u32(reinterpret_cast<const unsigned*>(abort))) return false;
    if ((long long)(globaltimer_ns() - t0) > limit_ns) return false;
  }
  return false;
}

// The instance parameters of the current item (copied from the workspace
// by the block), at file scope so that the item functions below read them
// from shared memory.
__shared__ FitParams<double> g_sp;
__shared__ CompState g_scs;

// The work of one item, each in a function of its own (not inlined), so that
// the tile march keeps the register allocation of the one-grid kernel
// instead of sharing it with the step and phase loops around it.
// CT: the instance's compensation words come by TMA (Nx % 8 == 0); TW:
// its tile width.
template <typename IdT, bool SIG, int MODE, bool CT, int TW>
__device__ __noinline__ bool batch_tile(const CompMaps* maps, long long t, int a, int b) {
  extern __shared__ __align__(128) unsigned char sm_raw[];
  return comp_tile<IdT, SIG, MODE, CT ? 1 : 0, true, TW>(g_sp, g_scs, *maps, t, b >> 16,
                                                         a & 0xffff, a >> 16, b & 0xffff, CT,
                                                         sm_raw);
}
// one whole z-boundary plane per item: warps take rows, lanes columns
__device__ __noinline__ void batch_shell(int kind, int plane, long long t) {
  const int Nx = g_sp.Nx, Ny = g_sp.Ny;
  Cell c;
  c.k = plane < 2 ? plane : g_sp.Nz - 4 + plane;
  for (int j = threadIdx.x >> 5; j < Ny; j += cThreads / 32) {
    c.j = j;
    for (int i = threadIdx.x & 31; i < Nx; i += 32) {
      c.i = i;
      if (kind == 1) comp_shell_h(g_sp, g_scs, c);
      else comp_shell_e(g_sp, g_scs, c, t);
    }
  }
}

template <typename IdT, bool SIG, int MODE>
__global__ void __launch_bounds__(cThreads, 2) k_batch_comp(const __grid_constant__ BatchArgs a) {
  __shared__ unsigned s_it;
  const int tid = threadIdx.x;
  const long long base = a.step0 + (a.step_dev ? *a.step_dev : 0);
  const unsigned per_step = (unsigned)(a.n_items[0] + a.n_items[1]);
  const unsigned total = per_step * (unsigned)a.n_steps;
  for (;;) {
    __syncthreads();   // the previous item is done with s_it, g_sp and g_scs
    if (tid == 0) s_it = atomicAdd(&a.sync->ticket, 1u);
    __syncthreads();
    const unsigned it = s_it;
    if (it >= total) break;
    const unsigned s = it / per_step, r = it - s * per_step;
    const int ph = r < (unsigned)a.n_items[0] ? 0 : 1;
    const BatchItem w = ph ? a.items[1][r - a.n_items[0]] : a.items[0][r];
    const BatchInst& I = a.insts[w.inst];
    // phase A of step s needs all of the instance's work of step s-1; phase
    // B of step s needs its phase-A items of step s
    int ok = 1;
    if (tid == 0)
      ok = wait_done(a.done + 2 * w.inst, (s + (unsigned)ph) * I.nA, s * I.nB, &a.sync->abort,
                     a.wait_ns);
    if (!__syncthreads_and(ok)) {
      if (tid == 0) {
        if (!ld_acquire_u32(reinterpret_cast<const unsigned*>(&a.sync->abort)) && I.p.status)
          atomicExch(I.p.status, 1);
        atomicExch(&a.sync->abort, 1);
      }
      return;
    }
    const long long t = base + s;
    const int par = (I.par_ref + (int)((t - I.t_ref) & 1)) & 1;
    {
      const uint64_t* src = reinterpret_cast<const uint64_t*>(&I.p);
      uint64_t* dst = reinterpret_cast<uint64_t*>(&g_sp);
      for (int q = tid; q < (int)(sizeof(FitParams<double>) / 8); q += cThreads)
        dst[q] = src[q];
      if (tid < (int)(sizeof(CompState) / 8))
        reinterpret_cast<uint64_t*>(&g_scs)[tid] =
            reinterpret_cast<const uint64_t*>(&I.cs[par])[tid];
    }
    __syncthreads();
    bool good = true;
    const CompMaps* maps = &a.maps[2 * w.inst + par];
    if (w.kind != 0) batch_shell(w.kind, w.a, t);
    else if (I.ct)
      good = I.tw == 32 ? batch_tile<IdT, SIG, MODE, true, 32>(maps, t, w.a, w.b)
                        : batch_tile<IdT, SIG, MODE, true, 64>(maps, t, w.a, w.b);
    else
      good = I.tw == 32 ? batch_tile<IdT, SIG, MODE, false, 32>(maps, t, w.a, w.b)
                        : batch_tile<IdT, SIG, MODE, false, 64>(maps, t, w.a, w.b);
    if (!good) {
      if (tid == 0) atomicExch(&a.sync->abort, 1);
      return;
    }
    // publish: this thread's global writes become visible to the TMA loads
    // (async proxy) and plain loads of the blocks that wait for the count
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      atomicAdd(a.done + 2 * w.inst + ph, 1u);
    }
  }
}

// The launch-per-phase form: each kernel runs one list of items of one
// step, block b item b of the list; the stream orders the lists (tiles and
// H rows of the boundary planes, then their E rows).  The instance
// parameters are read where they lie (read-only for the launch), and each
// kernel holds one kind of work, so the tile march keeps the registers of
// the one-grid kernel.
template <typename IdT, bool SIG, int MODE, bool CT, int TW>
__global__ void __launch_bounds__(cThreads, 2)
k_batch_tiles(const __grid_constant__ BatchArgs a, const BatchInst* __restrict__ insts,
              const BatchItem* __restrict__ list, int s) {
  extern __shared__ __align__(128) unsigned char sm_raw[];
  const long long t = a.step0 + s + (a.step_dev ? *a.step_dev : 0);
  const BatchItem w = list[blockIdx.x];
  const BatchInst& I = insts[w.inst];
  const int par = (I.par_ref + (int)((t - I.t_ref) & 1)) & 1;
  comp_tile<IdT, SIG, MODE, CT ? 1 : 0, false, TW>(I.p, I.cs[par], a.maps[2 * w.inst + par],
                                                   t, w.b >> 16, w.a & 0xffff, w.a >> 16,
                                                   w.b & 0xffff, CT, sm_raw);
}

__global__ void __launch_bounds__(cThreads)
k_batch_shells(const __grid_constant__ BatchArgs a, const BatchInst* __restrict__ insts,
               const BatchItem* __restrict__ list, int s) {
  const long long t = a.step0 + s + (a.step_dev ? *a.step_dev : 0);
  const BatchItem w = list[blockIdx.x];
  const BatchInst& I = insts[w.inst];
  const int par = (I.par_ref + (int)((t - I.t_ref) & 1)) & 1;
  const FitParams<double>& p = I.p;
  const CompState& cs = I.cs[par];
  Cell c;
  c.k = w.a < 2 ? w.a : p.Nz - 4 + w.a;
  for (int j = threadIdx.x >> 5; j < p.Ny; j += cThreads / 32) {
    c.j = j;
    for (int i = threadIdx.x & 31; i < p.Nx; i += 32) {
      c.i = i;
      if (w.kind == 1) comp_shell_h(p, cs, c);
      else comp_shell_e(p, cs, c, t);
    }
  }
}

// id width {1, 2} x J mode {0, sigma E} x face mode {1, 2}
constexpr int kBatchVariants = 8;
using BatchKern = void (*)(const BatchArgs);
const BatchKern kBatchKerns[kBatchVariants] = {
    k_batch_comp<uint8_t, false, 1>,  k_batch_comp<uint8_t, true, 1>,
    k_batch_comp<uint16_t, false, 1>, k_batch_comp<uint16_t, true, 1>,
    k_batch_comp<uint8_t, false, 2>,  k_batch_comp<uint8_t, true, 2>,
    k_batch_comp<uint16_t, false, 2>, k_batch_comp<uint16_t, true, 2>};
using TileKern = void (*)(const BatchArgs, const BatchInst*, const BatchItem*, int);
#define WK_BATCH_TILES(CT, TW)                                                                  \
  {k_batch_tiles<uint8_t, false, 1, CT, TW>,  k_batch_tiles<uint8_t, true, 1, CT, TW>,          \
   k_batch_tiles<uint16_t, false, 1, CT, TW>, k_batch_tiles<uint16_t, true, 1, CT, TW>,         \
   k_batch_tiles<uint8_t, false, 2, CT, TW>,  k_batch_tiles<uint8_t, true, 2, CT, TW>,          \
   k_batch_tiles<uint16_t, false, 2, CT, TW>, k_batch_tiles<uint16_t, true, 2, CT, TW>}
// [list]: TMA-word 64x8 tiles, TMA-word 32x16, other 64x8, other 32x16
const TileKern kTileKerns[4][kBatchVariants] = {WK_BATCH_TILES(true, 64), WK_BATCH_TILES(true, 32),
                                                WK_BATCH_TILES(false, 64),
                                                WK_BATCH_TILES(false, 32)};
#undef WK_BATCH_TILES
constexpr int kTileLists = 4;
// dynamic shared memory of the batched kernels: the larger tile layout
constexpr int kBatchSmem = CLayout<true, true, 64>::bytes > CLayout<true, true, 32>::bytes
                               ? CLayout<true, true, 64>::bytes
                               : CLayout<true, true, 32>::bytes;
bool g_tile_attr[kTileLists][kBatchVariants][64];
int g_batch_per_sm[kBatchVariants][64];
int g_batch_sms[kBatchVariants][64];
bool g_batch_attr[kBatchVariants][64];

constexpr size_t align_up(size_t b, size_t a) { return (b + a - 1) / a * a; }

struct Layout {
  size_t sync, insts, maps, items_a, items_b, total;
};
// [sync, counters][instances][maps][items A][items B]; the first region
// (everything before `insts`) is zeroed by every run
Layout batch_layout(int n_inst, size_t na, size_t nb) {
  Layout L;
  L.sync = 0;
  L.insts = align_up(sizeof(BatchSync) + 2 * sizeof(unsigned) * (size_t)n_inst, 128);
  L.maps = align_up(L.insts + n_inst * sizeof(BatchInst), 128);
  L.items_a = align_up(L.maps + 2 * (size_t)n_inst * sizeof(CompMaps), 128);
  L.items_b = align_up(L.items_a + na * sizeof(BatchItem), 128);
  L.total = align_up(L.items_b + nb * sizeof(BatchItem), 128);
  return L;
}

// Planes per tile item when the descriptor gives none.
constexpr int kBatchDefaultKC = 24;

// Checks every descriptor, forms the work lists and the variant; fills
// `insts` (parameters and state only; maps are encoded by the caller).
// Phase A lists the tiles of the instances whose compensation words come by
// TMA (64x8, then 32x16), then the other tiles (64x8, then 32x16), then the
// H rows of the boundary planes (parts[0..4] items each); phase B the E rows
// of the boundary planes.
int batch_build(const wk_fit_desc* descs, int n_inst, long long t_ref, const char* where,
                std::vector<BatchInst>* insts, std::vector<BatchItem>* ia,
                std::vector<BatchItem>* ib, int* variant, int* parts) {
  if (!descs) return wk_fail(WK_E_NULL, "%s: descs is NULL", where);
  if (n_inst < 1 || n_inst > (1 << 20)) return wk_fail(WK_E_RANGE, "%s: n_inst %d", where, n_inst);
  int var = -1;
  std::vector<BatchItem> tiles[kTileLists], shells_a;
  for (int q = 0; q < n_inst; q++) {
    const wk_fit_desc* d = &descs[q];
    int rc = wk_validate_fit(d, where);
    if (rc) return rc;
    if (d->dtype != WK_F32C)
      return wk_fail(WK_E_DTYPE, "%s: instance %d: dtype must be WK_F32C", where, q);
    if (!d->Ec[0] || !d->Ec[1] || !d->Hc[0] || !d->Hc[1])
      return wk_fail(WK_E_NULL, "%s: instance %d: compensation buffers missing", where, q);
    if (d->j_mode == WK_J_ARRAY)
      return wk_fail(WK_E_MODE, "%s: instance %d: WK_J_ARRAY is not available", where, q);
    if (d->step_dev)
      return wk_fail(WK_E_MODE, "%s: instance %d: step_dev is set per run, not per instance",
                     where, q);
    if (d->comp_stencil)
      return wk_fail(WK_E_MODE, "%s: instance %d: the compensated stencil runs the two-pass "
                                "kernels, not the batched launch", where, q);
    FitParams<double> p = make_params<double>(d, d->par);
    if (!tma_comp_supported(d, p))
      return wk_fail(WK_E_SHAPE, "%s: instance %d: needs Nx %% 4 == 0, dims >= 5, at most 64 "
                                 "materials and aligned buffers", where, q);
    const int mode = tma_comp_mode(p);
    if (mode == 0)
      return wk_fail(WK_E_MODE, "%s: instance %d: the x and y faces must be PEC-masked", where,
                     q);
    if (d->id_bytes > 2)
      return wk_fail(WK_E_DTYPE, "%s: instance %d: id_bytes must be 1 or 2", where, q);
    if (d->tile_rows != 0 && d->tile_rows != 8 && d->tile_rows != 16)
      return wk_fail(WK_E_RANGE, "%s: instance %d: tile_rows %d (0, 8 or 16)", where, q,
                     d->tile_rows);
    const int tw = d->tile_rows == 8 ? 64 : 32;
    const int v = (mode - 1) * 4 + (d->id_bytes - 1) * 2 + (d->j_mode == WK_J_SIGMA_E ? 1 : 0);
    if (var >= 0 && v != var)
      return wk_fail(WK_E_MODE, "%s: instance %d differs from instance 0 in face mode, id width "
                                "or J mode", where, q);
    var = v;
    BatchInst I;
    memset(&I, 0, sizeof(I));
    I.p = p;
    I.cs[0] = comp_state(d, 0);
    I.cs[1] = comp_state(d, 1);
    I.t_ref = t_ref;
    I.par_ref = d->par;
    I.tw = tw;
    I.ct = (p.Nx % 8 == 0 && ((uintptr_t)d->Hc[0] % 16) == 0 && ((uintptr_t)d->Hc[1] % 16) == 0 &&
            ((uintptr_t)d->Ec[0] % 16) == 0 && ((uintptr_t)d->Ec[1] % 16) == 0)
               ? 1
               : 0;
    insts->push_back(I);
    // tiles: the whole grid (MODE 1) or all of x and y for 2 <= k <= Nz-3
    int KC = d->tile_planes > 0 ? d->tile_planes : kBatchDefaultKC;
    const int planes = mode == 1 ? d->Nz : d->Nz - 4;
    if (KC > planes) KC = planes;
    if (KC > 32767) KC = 32767;
    const int tx = tw, ty = 512 / tw;
    const int gx = (d->Nx + tx - 1) / tx, gy = (d->Ny + ty - 1) / ty;
    const int gz = (planes + KC - 1) / KC;
    if (gx > 32767 || gy > 32767 || gz > 32767)
      return wk_fail(WK_E_SHAPE, "%s: instance %d: too many tiles", where, q);
    insts->back().nA = (unsigned)(gx * gy * gz + (mode == 2 ? 4 : 0));
    insts->back().nB = mode == 2 ? 4u : 0u;
    std::vector<BatchItem>* tl = &tiles[(I.ct ? 0 : 2) + (tw == 32 ? 1 : 0)];
    for (int bz = 0; bz < gz; bz++)
      for (int by = 0; by < gy; by++)
        for (int bx = 0; bx < gx; bx++)
          tl->push_back(BatchItem{q, 0, bx | (by << 16), bz | (KC << 16)});
    if (mode == 2) {
      for (int pl = 0; pl < 4; pl++) {
        shells_a.push_back(BatchItem{q, 1, pl, 0});
        ib->push_back(BatchItem{q, 2, pl, 0});
      }
    }
  }
  for (int l = 0; l < kTileLists; l++) {
    parts[l] = (int)tiles[l].size();
    ia->insert(ia->end(), tiles[l].begin(), tiles[l].end());
  }
  parts[kTileLists] = (int)shells_a.size();
  // the small shell items last, where they fill the tail of the phase
  ia->insert(ia->end(), shells_a.begin(), shells_a.end());
  *variant = var;
  return WK_OK;
}

}  // namespace

}  // namespace wk

using namespace wk;

extern "C" long long wk_batch_workspace_bytes(const wk_fit_desc* descs, int n_inst) {
  std::vector<BatchInst> insts;
  std::vector<BatchItem> ia, ib;
  int var = 0, parts[kTileLists + 1];
  if (batch_build(descs, n_inst, 0, "wk_batch_workspace_bytes", &insts, &ia, &ib, &var, parts))
    return -1;
  return (long long)batch_layout(n_inst, ia.size(), ib.size()).total;
}

extern "C" int wk_batch_prepare(const wk_fit_desc* descs, int n_inst, long long t_ref,
                                void* workspace, long long workspace_bytes, wk_batch_plan* plan,
                                void* stream) {
  const char* where = "wk_batch_prepare";
  if (!workspace || !plan) return wk_fail(WK_E_NULL, "%s: workspace or plan is NULL", where);
  if ((uintptr_t)workspace % 128)
    return wk_fail(WK_E_ALIGN, "%s: workspace must be 128-byte aligned", where);
  std::vector<BatchInst> insts;
  std::vector<BatchItem> ia, ib;
  int var = 0, parts[kTileLists + 1];
  int rc = batch_build(descs, n_inst, t_ref, where, &insts, &ia, &ib, &var, parts);
  if (rc) return rc;
  if (ia.size() > (size_t)INT32_MAX || ib.size() > (size_t)INT32_MAX)
    return wk_fail(WK_E_SHAPE, "%s: too many work items", where);
  const Layout L = batch_layout(n_inst, ia.size(), ib.size());
  if (workspace_bytes < (long long)L.total)
    return wk_fail(WK_E_RANGE, "%s: workspace of %lld bytes, %lld needed", where,
                   workspace_bytes, (long long)L.total);
  // host image of the workspace
  std::vector<unsigned char> img(L.total, 0);
  memcpy(img.data() + L.insts, insts.data(), insts.size() * sizeof(BatchInst));
  CompMaps* maps = reinterpret_cast<CompMaps*>(img.data() + L.maps);
  for (int q = 0; q < n_inst; q++) {
    const wk_fit_desc* d = &descs[q];
    const bool w32 = insts[q].tw == 32;
    const int ebx = w32 ? CGeom<true, 32>::ebx : CGeom<true, 64>::ebx;
    const int hbx = w32 ? CGeom<true, 32>::hbx : CGeom<true, 64>::hbx;
    const int cbx = w32 ? CGeom<true, 32>::cbx : CGeom<true, 64>::cbx;
    const int by = w32 ? CShape<32>::BY : CShape<64>::BY;
    const int hby = w32 ? CShape<32>::HBY : CShape<64>::HBY;
    for (int par = 0; par < 2; par++) {
      const CompState cs = comp_state(d, par);
      CompMaps& m = maps[2 * q + par];
      for (int c = 0; c < 3; c++) {
        const long long N = insts[q].p.N;
        if (!encode_3d(&m.e[c], cs.E_in + c * N, 4, d->Nx, d->Ny, d->Nz, ebx, by) ||
            !encode_3d(&m.h[c], cs.H_in + c * N, 4, d->Nx, d->Ny, d->Nz, hbx, hby))
          return wk_fail(WK_E_SHAPE, "%s: instance %d: tensor map encoding failed", where, q);
        if (insts[q].ct &&
            (!encode_3d(&m.c[c], cs.Hc_in + c * N, 2, d->Nx, d->Ny, d->Nz, cbx, hby) ||
             !encode_3d(&m.c[3 + c], cs.Ec_in + c * N, 2, d->Nx, d->Ny, d->Nz, cbx, hby)))
          return wk_fail(WK_E_SHAPE, "%s: instance %d: tensor map encoding failed", where, q);
      }
    }
  }
  if (!ia.empty()) memcpy(img.data() + L.items_a, ia.data(), ia.size() * sizeof(BatchItem));
  if (!ib.empty()) memcpy(img.data() + L.items_b, ib.data(), ib.size() * sizeof(BatchItem));
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return wk_fail(-(int)e, "%s: %s", where, cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return wk_fail(WK_E_RANGE, "%s: device %d", where, dev);
  const int smem = kBatchSmem;
  const BatchKern kern = kBatchKerns[var];
  if (!g_batch_attr[var][dev]) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
      e = cudaDeviceGetAttribute(&g_batch_sms[var][dev], cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_batch_per_sm[var][dev], kern, cThreads,
                                                        smem);
    if (e != cudaSuccess) return wk_fail(-(int)e, "%s: %s", where, cudaGetErrorString(e));
    if (g_batch_per_sm[var][dev] < 1)
      return wk_fail(WK_E_SHAPE, "%s: the batched kernel does not fit on an SM", where);
    g_batch_attr[var][dev] = true;
  }
  for (int l = 0; l < kTileLists; l++) {
    if (g_tile_attr[l][var][dev]) continue;
    e = cudaFuncSetAttribute(kTileKerns[l][var], cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
    if (e != cudaSuccess) return wk_fail(-(int)e, "%s: %s", where, cudaGetErrorString(e));
    g_tile_attr[l][var][dev] = true;
  }
  cudaStream_t st = (cudaStream_t)stream;
  e = cudaMemcpyAsync(workspace, img.data(), L.total, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);   // the host image dies with this call
  if (e != cudaSuccess) return wk_fail(-(int)e, "%s: %s", where, cudaGetErrorString(e));
  memset(plan, 0, sizeof(*plan));
  plan->workspace = workspace;
  plan->workspace_bytes = (long long)L.total;
  plan->n_inst = n_inst;
  plan->n_items[0] = (int)ia.size();
  plan->n_items[1] = (int)ib.size();
  plan->grid = g_batch_sms[var][dev] * g_batch_per_sm[var][dev];
  plan->smem = smem;
  plan->variant = var;
  plan->device = dev;
  plan->offsets[0] = (long long)L.insts;
  plan->offsets[1] = (long long)L.maps;
  plan->offsets[2] = (long long)L.items_a;
  plan->offsets[3] = (long long)L.items_b;
  for (int q = 0; q <= kTileLists; q++) plan->n_parts[q] = parts[q];
  plan->form = WK_BATCH_PERSISTENT;
  return WK_OK;
}

extern "C" int wk_batch_run(const wk_batch_plan* plan, int n_steps, long long step0,
                            const long long* step_dev, long long wait_ns, void* stream) {
  const char* where = "wk_batch_run";
  if (!plan || !plan->workspace) return wk_fail(WK_E_NULL, "%s: plan or workspace is NULL", where);
  if (plan->variant < 0 || plan->variant >= kBatchVariants || plan->grid < 1)
    return wk_fail(WK_E_MODE, "%s: plan was not filled by wk_batch_prepare", where);
  if (n_steps < 0) return wk_fail(WK_E_RANGE, "%s: n_steps %d", where, n_steps);
  if (n_steps == 0) return WK_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return wk_fail(-(int)e, "%s: %s", where, cudaGetErrorString(e));
  if (dev != plan->device)
    return wk_fail(WK_E_MODE, "%s: plan prepared on device %d, current device %d", where,
                   plan->device, dev);
  unsigned char* ws = static_cast<unsigned char*>(plan->workspace);
  BatchArgs a;
  memset(&a, 0, sizeof(a));
  a.sync = reinterpret_cast<BatchSync*>(ws);
  a.insts = reinterpret_cast<const BatchInst*>(ws + plan->offsets[0]);
  a.maps = reinterpret_cast<const CompMaps*>(ws + plan->offsets[1]);
  a.items[0] = reinterpret_cast<const BatchItem*>(ws + plan->offsets[2]);
  a.items[1] = reinterpret_cast<const BatchItem*>(ws + plan->offsets[3]);
  a.n_items[0] = plan->n_items[0];
  a.n_items[1] = plan->n_items[1];
  a.n_steps = n_steps;
  a.step0 = step0;
  a.step_dev = step_dev;
  a.done = reinterpret_cast<unsigned*>(ws + sizeof(BatchSync));
  a.wait_ns = wait_ns > 0 ? wait_ns : kDepNs;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->form == WK_BATCH_PHASES) {
    // the tile lists and the boundary-plane H rows of phase A, then phase B
    const BatchItem* lists[kTileLists + 2];
    int counts[kTileLists + 2];
    const BatchItem* at = a.items[0];
    for (int l = 0; l <= kTileLists; l++) {
      lists[l] = at;
      counts[l] = plan->n_parts[l];
      at += counts[l];
    }
    lists[kTileLists + 1] = a.items[1];
    counts[kTileLists + 1] = plan->n_items[1];
    timer_begin(st);
    for (int s = 0; s < n_steps; s++) {
      for (int l = 0; l < kTileLists + 2; l++) {
        if (counts[l] == 0) continue;
        if (l < kTileLists)
          kTileKerns[l][plan->variant]<<<counts[l], cThreads, plan->smem, st>>>(a, a.insts,
                                                                              lists[l], s);
        else
          k_batch_shells<<<counts[l], cThreads, 0, st>>>(a, a.insts, lists[l], s);
      }
    }
    timer_end(st);
    return wk_check_launch(where);
  }
  if (plan->form != WK_BATCH_PERSISTENT)
    return wk_fail(WK_E_MODE, "%s: form %d", where, plan->form);
  const long long per_step_items = (long long)plan->n_items[0] + plan->n_items[1];
  if ((long long)per_step_items * n_steps >= (1LL << 32))
    return wk_fail(WK_E_RANGE, "%s: %d steps of %lld items exceed the ticket range", where,
                   n_steps, per_step_items);
  // the ticket, the abort flag and the completion counters start at zero
  // on every run (a run that gave up leaves them set)
  e = cudaMemsetAsync(ws, 0, (size_t)plan->offsets[0], st);
  if (e != cudaSuccess) return wk_fail(-(int)e, "%s: %s", where, cudaGetErrorString(e));
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3((unsigned)plan->grid);
  cfg.blockDim = dim3(cThreads);
  cfg.dynamicSmemBytes = (size_t)plan->smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  timer_begin(st);
  e = cudaLaunchKernelEx(&cfg, kBatchKerns[plan->variant], a);
  timer_end(st);
  if (e != cudaSuccess) return wk_fail(-(int)e, "%s: %s", where, cudaGetErrorString(e));
  return wk_check_launch(where);
}
