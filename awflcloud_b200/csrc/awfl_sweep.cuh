// The line-sweep kernel skeleton shared by the FP64 and FP32 forms.
//
// A CTA owns W whole lines along the sweep direction DIR and marches along them in
// chunks of C cells. Because no other CTA touches those lines, the tendency can be
// applied in place (MODE_APPLY) with no race: every stencil value a chunk reads comes
// from a shared-memory ring holding the ORIGINAL values of positions
// [base-HS, base+C+HS), refilled one chunk ahead of the updates, and the first HS rows
// (needed again by the periodic wrap at the end of the line) are saved before they are
// overwritten.
//
// Per chunk: (A) the chunk's ring rows are in place (landed by TMA or cp.async, or stored
// from registers); the next chunk's rows are requested; reconstruct cells base..base+C-1
// -> left/right edge states; Riemann flux at their left faces (the left state of the
// first face is carried from the previous chunk); divergence and update of cells
// base-1..base+C-2 (the last cell's right face is computed in the next chunk). Where a
// line's C cells are consecutive lanes of one warp (SHFL) the edge states and fluxes move
// between neighbouring cells by warp shuffles and (A) is the chunk's only CTA barrier;
// otherwise they go through shared memory with barriers (B), (C), (D) between the steps.
// The last cell of the line is finished after the loop.
//
// Boundary handling reproduces the reference's halo fill (Spatial_euler3d_cons_expl_
// cart_fv_Agrid.h:631-662, 994-1025, 1351-1382) and edge-value BCs (:816-837, 1176-1197,
// 1557-1578): periodic wraps; a wall copies the edge cell with zero normal momentum, and
// its boundary face uses the interior state on both sides. The halo values are also
// written to the state's halo cells, as the reference does in place.
// An x sweep of a slab of a larger grid (A.xh[side] != nullptr) takes an end's halo
// values from the neighbouring slab's columns instead (hs+1 of them: the neighbour's edge
// cell is reconstructed here, so the face between the slabs gets the same left and right
// states, hence the same flux, as in the undivided grid).
//
// The physics policy P supplies the element type, the per-cell reconstruction (+ADER +
// time average), the face flux, the tendency and the in-place update:
//   using Real; using Args;                         Args has state/tend/nx/ny/nz/bc/mode/sim2d
//   template <int ORD, int DIR, class S> recon(sten, kb, A, eL[5], eR[5], src, cell)
//                                          (cell: the cell's (k,j,i) index, -1 for the
//                                          periodic prologue's repeat of cell L-1)
//   template <int DIR, int NG>            flux(qL[5], qR[5], kf, A, F[5])
//                                          (kf: the face's k for z, the line's k for x, y)
//   template <int DIR>                    tendency(v, Fl, Fr, src, A) -> Real
//   struct Aux; load_aux(A, g0, sv, aux)   per-cell inputs of the update (variable v at
//                                          g0 + v*sv), loaded a reconstruction ahead
//   apply(A, gidx, orig, tnd, aux, v)      state[gidx] = orig "+" dt*tnd (MODE_APPLY)
//   kAsyncRing                             next-chunk rows by cp.async into a 4C ring
//   kTmaRing, prepare_tma(A, ord, dir, C, W) (host), tma_map(A), tma_map_global(a, g),
//   flag_timeout(A)                        next-chunk rows of interior chunks by tiled TMA
//                                          boxes through a tensor map (kernel parameter
//                                          for single-grid sweeps, the work list in
//                                          global memory for ensembles)
//   min_blocks(ORD)                        CTAs per SM the register budget must allow
//   kSlab                                  the policy runs x splits of slabs (A.xh)
//   load(A, gidx) / store(A, gidx, x)      state element access (halo writes)
//   store_tend(A, tidx, x)                 tendency output (MODE_TEND)
#pragma once

#include <type_traits>

#include "awfl_internal.h"

namespace awfl {

// Asynchronous global -> shared copy of one element (cp.async, sm_80+; 4 or 8 bytes).
template <class T> __device__ __forceinline__ void cp_async_row(T *dst_smem, const T *src_gmem) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "cp.async of 4 or 8 bytes");
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src_gmem), "n"(sizeof(T)) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Tiled TMA loads (cp.async.bulk.tensor) completing on a shared-memory mbarrier. The
// destination is the CTA's own shared memory (128-byte aligned boxes), the source this
// GPU's global memory through a tensor map held in the kernel parameter; no multicast.
__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *mb, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(mb)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_inval(unsigned long long *mb) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_addr(mb)) : "memory");
}
__device__ __forceinline__ void mbar_arm(unsigned long long *mb, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(mb)), "r"(bytes) : "memory");
}
// Waits for the phase of the given parity, giving up after a bounded number of polls
// (each poll may suspend the thread for a while); returns false then.
__device__ __forceinline__ bool mbar_wait(unsigned long long *mb, unsigned parity) {
  const unsigned a = smem_addr(mb);
  for (int i = 0; i < (1 << 20); i++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// One 3-D box of the tensor map at element coordinates (x, y, z) into shared memory.
__device__ __forceinline__ void tma_load_3d(void *dst_smem, const void *tmap, int x, int y, int z,
                                            unsigned long long *mb) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_addr(dst_smem)),
      "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_addr(mb))
      : "memory");
}
// Warp shuffle up by `delta` lanes within segments of `width` lanes, for a value of any
// type made of 4-byte words (float, double, a dual number); every lane of the warp calls it.
template <class T> __device__ __forceinline__ T shfl_up_any(const T &x, int delta, int width) {
  static_assert(sizeof(T) % 4 == 0, "shuffled types are made of 4-byte words");
  constexpr int N = (int)(sizeof(T) / 4);
  unsigned u[N];
  __builtin_memcpy(u, &x, sizeof(T));
#pragma unroll
  for (int i = 0; i < N; i++) u[i] = __shfl_up_sync(0xffffffffu, u[i], delta, width);
  T y;
  __builtin_memcpy(&y, u, sizeof(T));
  return y;
}

// orders this thread's generic-proxy shared-memory accesses before later async-proxy ones
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// Row pitch (elements) of the ring of a y/z sweep fed by TMA: the box starts at the
// 16-byte-aligned x = bx*W of the halo-inclusive row (the tile's first line sits at
// column HS), spans at least W + HS columns in a multiple of 4, and a chunk's C rows
// (one box) are a multiple of 128 bytes so that every box lands 128-byte aligned.
__host__ __device__ constexpr int tma_ring_pitch_of(int ord, int C, int W, int esz) {
  int rw = (W + (ord - 1) / 2 + 3) / 4 * 4;
  while ((C * rw * esz) % 128 != 0) rw += 4;
  return rw;
}
template <int ORD, int C, int W, int ESZ> __host__ __device__ constexpr int tma_ring_pitch() {
  return tma_ring_pitch_of(ORD, C, W, ESZ);
}

// A policy with `static constexpr bool kFaceRec = true` sees every face the sweep computes:
// P::face_rec<ORD, DIR>(A, face, kf, qL, qR, F) with the face's index in the tracer path's
// face numbering (faces along DIR: n+1 per line), the k passed to the flux, the face's two
// states after the edge BCs and its flux (the tracer transport records them).
template <class P, class = void> struct PolicyFaceRec : std::false_type {};
template <class P> struct PolicyFaceRec<P, std::void_t<decltype(P::kFaceRec)>> : std::bool_constant<P::kFaceRec> {};

// One CTA's tile: lines bx*W .. bx*W+W-1 of plane `by` (x, y sweeps: by = k; z: by = j).
// tmap: the tensor map of the TMA path (a kernel-parameter or global address), or nullptr
// (the instantiation with TMA = true then stages every chunk by cp.async).
// SLAB: the x sweep of a slab of a larger grid, whose ends may take their halo values from
// the neighbouring slabs (A.xh); a separate instantiation, so that the plain sweeps carry
// none of its registers.
template <class P, int ORD, int DIR, int C, int W, bool TMA = false, bool SLAB = false>
__device__ __forceinline__ void sweep_tile(const typename P::Args &A, const int bx, const int by,
                                           const void *tmap = nullptr) {
  using Real = typename P::Real;
  constexpr int HS = (ORD - 1) / 2;
  constexpr int NG = OrdTraits<ORD>::NGLL;
  // Next-chunk rows: policies with kAsyncRing copy them global -> shared with cp.async one
  // chunk ahead (issued before the reconstruction, no registers held), which needs a ring
  // of 4C so that the rows in flight never share a slot with rows still being read;
  // otherwise they are loaded into registers and stored at the next chunk's start.
  constexpr bool ASYNC = P::kAsyncRing;
  constexpr int R = ASYNC ? 4 * C : 2 * C;  // ring length (power of two, >= C + 2*HS)
  // TMA path (TMA, with the async ring): a chunk whose rows are all interior arrives as
  // five tiled TMA boxes, one per variable, issued by one thread and completing on an
  // mbarrier -- x sweep: box {C positions, W lines}, landing as one page [W][C] of the
  // ring; y/z sweeps: box {RW columns from x = bx*W, C positions}, landing as C ring rows
  // of pitch RW with line w at column HS + w. Other chunks (and a tile whose wait gave
  // up) use cp.async. Out-of-range box elements (the last tile's missing lines) read as
  // zero and are never used.
  static_assert(!TMA || ASYNC, "the TMA path feeds the async ring");
  constexpr int RW = (TMA && DIR != 0) ? tma_ring_pitch<ORD, C, W, (int)sizeof(Real)>() : W;
  static_assert(!TMA || DIR != 0 || ((C * W * (int)sizeof(Real)) % 128 == 0 && (2 * HS * (int)sizeof(Real)) % 16 == 0 &&
                                     (C * (int)sizeof(Real)) % 16 == 0),
                "x-sweep TMA pages must be 128-byte multiples starting at 16-byte-aligned x");
  static_assert(!TMA || DIR == 0 || (W * (int)sizeof(Real)) % 16 == 0, "y/z-sweep TMA boxes start at x = bx*W");
  constexpr int NM = 1 + DIR;
  static_assert((C & (C - 1)) == 0 && C >= 2 * HS, "chunk must be a power of two >= 2*HS");
  // Register path: load the next chunk's rows before the reconstruction (latency hidden
  // behind it, at the cost of 5 live registers) for the z sweep, whose loads stride over
  // whole planes; after the updates for x and y, where occupancy matters more (measured).
  constexpr bool EARLY_PREFETCH = !ASYNC && DIR == 2;
  // The C cells of a chunk of one line are C consecutive lanes of one warp (x sweep: a
  // warp holds 32/C lines along x; y/z sweeps: 32/C neighbouring lines, so that a warp's
  // global accesses are 32/C consecutive x cells in each of C rows), so the interface
  // states, fluxes and z sources pass between neighbouring cells by warp shuffles (the
  // first cell's left neighbour is the previous chunk's last cell, carried per line in
  // shared memory); the chunk needs no CTA barrier besides the ring's (A). The y/z sweeps
  // of the register-staged path keep a warp along x across lines (32/W positions) and
  // trade through shared memory between barriers: a warp's next-chunk loads from global
  // memory would otherwise touch C rows instead of 32/W (FP64 z split measured 3.61 ->
  // 3.71 ms with the shuffles).
  constexpr bool SHFL = C <= 32 && (C * W) % 32 == 0 && (DIR == 0 || ASYNC);

  __shared__ __align__(128) Real ring[5][R * RW];
  __shared__ __align__(8) unsigned long long mbar;  // TMA path only
  __shared__ int sAbort;                            // TMA path: a wait of this tile gave up
  __shared__ Real sEL[5][(C + 1) * W];
  __shared__ Real sER[5][(C + 1) * W];
  __shared__ Real sF[5][(C + 1) * W];
  __shared__ Real sSrc[DIR == 2 ? (C + 1) * W : 1];
  __shared__ Real sWrap[5][HS * W];
  __shared__ Real sEL0[5][W];

  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  // position in chunk, line within CTA
  const int c = DIR == 0 ? (int)threadIdx.x : (SHFL ? (tid & (C - 1)) : (int)threadIdx.y);
  const int w = DIR == 0 ? (int)threadIdx.y : (SHFL ? tid / C : (int)threadIdx.x);
  // edge/flux slot (0..C) of this line: consecutive threads of a warp hit consecutive words
  auto E = [&](int slot) { return DIR == 0 ? w * (C + 1) + slot : slot * W + w; };

  const int nx = A.nx, ny = A.ny, nz = A.nz;
  const long sx = 1, sy = nx + 2 * HS, sz = (long)(ny + 2 * HS) * sy, sv = (long)(nz + 2 * HS) * sz;
  int L, kline = 0;
  bool valid;
  long lb;  // offset of (v=0, position 0 along DIR) of this line, halo-inclusive frame
  long sd;  // stride along DIR
  long tb;  // tendency offset of position 0
  long tsd;
  long fb, fsd;  // face index of position 0 and its stride along DIR (face records only)
  if (DIR == 0) {
    const int k = by, j = bx * W + w;
    L = nx; valid = j < ny; kline = k;
    lb = (HS + k) * sz + (HS + (valid ? j : 0)) * sy + HS * sx; sd = sx;
    tb = ((long)k * ny + (valid ? j : 0)) * nx; tsd = 1;
    fb = ((long)k * ny + (valid ? j : 0)) * (nx + 1); fsd = 1;
  } else if (DIR == 1) {
    const int k = by, i = bx * W + w;
    L = ny; valid = i < nx; kline = k;
    lb = (HS + k) * sz + HS * sy + HS + (valid ? i : 0); sd = sy;
    tb = (long)k * ny * nx + (valid ? i : 0); tsd = nx;
    fb = (long)k * (ny + 1) * nx + (valid ? i : 0); fsd = nx;
  } else {
    const int j = by, i = bx * W + w;
    L = nz; valid = i < nx;
    lb = HS * sz + (HS + j) * sy + HS + (valid ? i : 0); sd = sz;
    tb = (long)j * nx + (valid ? i : 0); tsd = (long)ny * nx;
    fb = (long)j * nx + (valid ? i : 0); fsd = (long)ny * nx;
  }
  const long tv = (long)nz * ny * nx;
  const bool periodic = A.bc == BC_PERIODIC;
  // x sweep of a slab: the ends bordering another slab, and that slab's columns
  // ([5][nz][ny][HS+1] per side: side 0 holds positions -(HS+1)..-1, side 1 L..L+HS)
  static_assert(!SLAB || DIR == 0, "slabs are cut along x");
  bool xlo = false, xhi = false;
  int jline = 0;
  if constexpr (SLAB) {
    xlo = A.xh[0] != nullptr;
    xhi = A.xh[1] != nullptr;
    jline = bx * W + w;
  }
  auto XH = [&](int side, int v, int col) -> Real {
    return Real(A.xh[side][(((long)v * nz + kline) * ny + jline) * (HS + 1) + col]);
  };

  auto G = [&](int v, int p) -> Real { return P::load(A, lb + v * sv + p * sd); };
  // ring slot of position p: the async ring counts from p = HS so that a chunk's rows
  // (positions base+HS .. base+C+HS-1) fill one aligned run of C slots. The x sweep's
  // async ring is paged: page s/C holds [line][slot % C], so the lines of a warp read
  // 32 consecutive words (no bank conflict) and a chunk is one TMA box.
  auto ringAt = [&](int v, int p) -> Real & {
    if constexpr (ASYNC) {
      const int s = (p - HS) & (R - 1);
      if constexpr (DIR == 0) return ring[v][(s / C) * (W * C) + w * C + (s & (C - 1))];
      else return ring[v][s * RW + (TMA ? HS : 0) + w];
    } else {
      const int s = p & (R - 1);
      return DIR == 0 ? ring[v][w * R + s] : ring[v][s * W + w];
    }
  };
  auto topval = [&](int v, int p, bool first) -> Real {  // p >= L
    const int q = p - L;
    if (q >= HS) return Real(0);  // beyond the last cell's stencil: never read
    if (xhi) return XH(1, v, q);
    if (periodic) return first ? G(v, q) : sWrap[v][q * W + w];
    return v == NM ? Real(0) : G(v, L - 1);
  };
  auto finish = [&](int cell, const Real *Fl, const Real *Fr, Real sa, const typename P::Aux &aux) {
#pragma unroll
    for (int v = 0; v < 5; v++) {
      const Real tnd = P::template tendency<DIR>(v, Fl[v], Fr[v], sa, A);
      if (A.mode == MODE_APPLY) P::apply(A, lb + v * sv + cell * sd, ringAt(v, cell), tnd, aux, v);
      else P::store_tend(A, tb + v * tv + cell * tsd, tnd);
    }
  };
  // a row value into its ring slot: asynchronously when it is a load of an interior cell
  auto stage = [&](int v, int p, bool first) {
    if constexpr (ASYNC) {
      if (p < L) cp_async_row(&ringAt(v, p), &A.state[lb + v * sv + p * sd]);
      else ringAt(v, p) = topval(v, p, first);
    }
  };
  // the chunk whose rows start at position p0 comes by TMA (uniform in the CTA)
  auto chunk_tma = [&](int p0) { return TMA && tmap != nullptr && p0 + C <= L; };
  constexpr unsigned kTmaBytes = 5u * C * (DIR == 0 ? W : RW) * (unsigned)sizeof(Real);
  auto issue_tma = [&](int p0) {  // thread 0 only
    if constexpr (TMA) {
      const int s0 = (p0 - HS) & (R - 1);  // a multiple of C
      const int zp = nz + 2 * HS;          // the map's z extent per variable
      mbar_arm(&mbar, kTmaBytes);
#pragma unroll
      for (int v = 0; v < 5; v++) {
        if (DIR == 0) tma_load_3d(&ring[v][(s0 / C) * (W * C)], tmap, HS + p0, HS + bx * W, v * zp + HS + by, &mbar);
        else if (DIR == 1) tma_load_3d(&ring[v][s0 * RW], tmap, bx * W, HS + p0, v * zp + HS + by, &mbar);
        else tma_load_3d(&ring[v][s0 * RW], tmap, bx * W, HS + by, v * zp + HS + p0, &mbar);
      }
    }
  };

  // ---- prologue: bottom halo, saved wrap rows, top halo; chunk-0 prefetch
  if (TMA && tid == 0) {
    mbar_init(&mbar, 1);
    sAbort = 0;
  }
  if (valid && c < HS) {
#pragma unroll
    for (int v = 0; v < 5; v++) {
      const Real bot = xlo ? XH(0, v, c + 1) : (periodic ? G(v, L + c - HS) : (v == NM ? Real(0) : G(v, 0)));
      const Real top = xhi ? XH(1, v, c) : (periodic ? G(v, c) : (v == NM ? Real(0) : G(v, L - 1)));
      // position c of a wall line shorter than HS is a top halo cell: its stencil value is
      // the wall copy (read from the interior, never from a halo cell another thread of
      // this prologue is writing); periodic lines are at least HS long (awfl_create)
      const Real orig = c < L ? G(v, c) : top;
      ringAt(v, c - HS) = bot;
      ringAt(v, c) = orig;
      sWrap[v][c * W + w] = orig;
      P::store(A, lb + v * sv + (c - HS) * sd, bot);
      P::store(A, lb + v * sv + (L + c) * sd, top);
    }
  }
  Real pre[ASYNC ? 1 : 5];
  bool cur_tma = false;  // this chunk's rows come by TMA (uniform in the CTA)
  unsigned phase = 0;    // TMA phases of the mbarrier issued so far
  if constexpr (TMA) {
    cur_tma = chunk_tma(HS);
    fence_proxy_async();  // the prologue's generic writes to ring slots before any TMA write
    __syncthreads();      // the mbarrier is initialised before its first use
    if (cur_tma && tid == 0) issue_tma(HS);
    if (cur_tma) phase++;
  }
  if (valid && !cur_tma) {
    const int p = HS + c;
    if constexpr (ASYNC) {
#pragma unroll
      for (int v = 0; v < 5; v++) stage(v, p, true);
    } else {
#pragma unroll
      for (int v = 0; v < 5; v++) pre[v] = p < L ? G(v, p) : topval(v, p, true);
    }
  }
  // periodic: the left state of face 0 is the right edge of cell L-1; a slab bordering
  // another below: the right edge of that slab's last cell (position -1)
  if (valid && (periodic || xlo) && c == 0) {
    auto wrapSten = [&](int v, int m) -> Real {
      if (xlo) {
        const int p = -1 - HS + m;
        return p < 0 ? XH(0, v, p + HS + 1) : G(v, p);
      }
      int p = L - 1 - HS + m;
      p %= L;
      if (p < 0) p += L;
      return G(v, p);
    };
    Real eL[5], eR[5], sa;
    P::template recon<ORD, DIR>(wrapSten, DIR == 2 ? L - 1 : kline, A, eL, eR, sa, -1L);
#pragma unroll
    for (int v = 0; v < 5; v++) sER[v][E(0)] = eR[v];
  }

  const int nchunk = (L + C - 1) / C;
  for (int t = 0; t < nchunk; t++) {
    const int base = t * C;
    const int nvalid = min(C, L - base);
    if constexpr (TMA) {
      // the chunk's boxes have landed; a wait that gives up flags the error and ends the
      // tile's use of TMA (the rest of the tile's chunks come by cp.async)
      if (cur_tma && !mbar_wait(&mbar, (phase - 1) & 1u)) {
        P::flag_timeout(A);
        sAbort = 1;
      }
      // (generic reads of a slot, then a TMA write into it after barrier (A): ordered by
      // the barrier. Generic writes into slots a TMA box later fills happen only in the
      // prologue -- fenced there -- or in the last chunks, after the tile's last box.)
    }
    if constexpr (ASYNC) {
      cp_async_wait_all();  // this thread's rows of the chunk have landed
    } else if (valid) {
#pragma unroll
      for (int v = 0; v < 5; v++) ringAt(v, base + HS + c) = pre[v];
    }
    __syncthreads();  // (A)
    if constexpr (ASYNC) {  // the next chunk's rows, a chunk ahead
      bool next_tma = false;
      if constexpr (TMA) {
        next_tma = t + 1 < nchunk && chunk_tma(base + C + HS) && !*(volatile int *)&sAbort;
        if (next_tma && tid == 0) issue_tma(base + C + HS);
        if (next_tma) phase++;
      }
      if (!next_tma && valid && t + 1 < nchunk) {
#pragma unroll
        for (int v = 0; v < 5; v++) stage(v, base + C + HS + c, false);
      }
      cur_tma = next_tma;
    }
    // the compensation (or other per-cell input) of the cell this thread updates below
    typename P::Aux aux;
    if (valid && c < nvalid && base + c >= 1 && A.mode == MODE_APPLY) P::load_aux(A, lb + (base + c - 1) * sd, sv, aux);
    // next chunk's rows (stored into the ring at the next (A); the updates of this chunk
    // never reach them)
    if (EARLY_PREFETCH && valid && t + 1 < nchunk) {
      const int p = base + C + HS + c;
#pragma unroll
      for (int v = 0; v < 5; v++) pre[v] = p < L ? G(v, p) : topval(v, p, false);
    }
    Real eL[5], eR[5], sa;
    if constexpr (SHFL) {  // defined values on the lanes that reconstruct nothing
#pragma unroll
      for (int v = 0; v < 5; v++) eL[v] = eR[v] = Real(0);
      sa = Real(0);
    }
    if (valid && c < nvalid) {
      const int p = base + c;
      auto sten = [&](int v, int m) -> Real { return ringAt(v, p - HS + m); };
      P::template recon<ORD, DIR>(sten, DIR == 2 ? p : kline, A, eL, eR, sa, tb + p * tsd);
      if constexpr (!SHFL) {
#pragma unroll
        for (int v = 0; v < 5; v++) {
          sEL[v][E(c)] = eL[v];
          sER[v][E(c + 1)] = eR[v];
        }
        if (DIR == 2) sSrc[E(c + 1)] = sa;
      }
      if (p == 0) {
#pragma unroll
        for (int v = 0; v < 5; v++) sEL0[v][w] = eL[v];
      }
    }
    if constexpr (SHFL) {
      const bool act = valid && c < nvalid;
      // face base+c: left state = right edge of cell base+c-1 (the lane below, or the carry)
      Real qL[5], F[5];
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const Real up = shfl_up_any(eR[v], 1, C);
        qL[v] = c == 0 ? sER[v][E(0)] : up;
      }
      if (act) {
        if (base + c == 0 && !periodic && !xlo) {
#pragma unroll
          for (int v = 0; v < 5; v++) qL[v] = eL[v];
        }
        P::template flux<DIR, NG>(qL, eL, DIR == 2 ? base + c : kline, A, F);
        if constexpr (PolicyFaceRec<P>::value)
          P::template face_rec<ORD, DIR>(A, fb + (base + c) * fsd, DIR == 2 ? base + c : kline, qL, eL, F);
      } else {
#pragma unroll
        for (int v = 0; v < 5; v++) F[v] = Real(0);
      }
      // cell base+c-1: its left face's flux from the lane below (or the carry), its right
      // face's from this lane
      Real Fl[5];
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const Real up = shfl_up_any(F[v], 1, C);
        Fl[v] = c == 0 ? sF[v][E(0)] : up;
      }
      Real sl = Real(0);  // z: the source term of cell base+c-1
      if constexpr (DIR == 2) {
        const Real up = shfl_up_any(sa, 1, C);
        sl = c == 0 ? sSrc[E(0)] : up;
      }
      if (act && base + c >= 1) finish(base + c - 1, Fl, F, sl, aux);
      if (!ASYNC && valid && t + 1 < nchunk) {
        const int p = base + C + HS + c;
#pragma unroll
        for (int v = 0; v < 5; v++) pre[v] = p < L ? G(v, p) : topval(v, p, false);
      }
      __syncwarp();  // the line's reads of its ring rows and carry are done
      if (valid && c == nvalid - 1) {  // the carry: last cell's right edge, right-face flux, source
#pragma unroll
        for (int v = 0; v < 5; v++) {
          sER[v][E(0)] = eR[v];
          sF[v][E(0)] = F[v];
        }
        if (DIR == 2) sSrc[E(0)] = sa;
      }
      __syncwarp();
      continue;
    }
    __syncthreads();  // (B)
    if (valid && c < nvalid) {
      const int f = base + c;  // face index = left face of cell f
      Real qL[5], qR[5], F[5];
#pragma unroll
      for (int v = 0; v < 5; v++) qR[v] = sEL[v][E(c)];
#pragma unroll
      for (int v = 0; v < 5; v++) qL[v] = (f == 0 && !periodic && !xlo) ? qR[v] : sER[v][E(c)];
      P::template flux<DIR, NG>(qL, qR, DIR == 2 ? f : kline, A, F);
      if constexpr (PolicyFaceRec<P>::value) P::template face_rec<ORD, DIR>(A, fb + f * fsd, DIR == 2 ? f : kline, qL, qR, F);
#pragma unroll
      for (int v = 0; v < 5; v++) sF[v][E(c + 1)] = F[v];
    }
    __syncthreads();  // (C)
    if (valid && c < nvalid) {
      const int cell = base + c - 1;
      if (cell >= 0) {
        Real Fl[5], Fr[5];
#pragma unroll
        for (int v = 0; v < 5; v++) {
          Fl[v] = sF[v][E(c)];
          Fr[v] = sF[v][E(c + 1)];
        }
        finish(cell, Fl, Fr, DIR == 2 ? sSrc[E(c)] : Real(0), aux);
      }
    }
    if (!ASYNC && !EARLY_PREFETCH && valid && t + 1 < nchunk) {
      const int p = base + C + HS + c;
#pragma unroll
      for (int v = 0; v < 5; v++) pre[v] = p < L ? G(v, p) : topval(v, p, false);
    }
    __syncthreads();  // (D)
    if (valid && c == 0) {
#pragma unroll
      for (int v = 0; v < 5; v++) {
        sER[v][E(0)] = sER[v][E(nvalid)];
        sF[v][E(0)] = sF[v][E(nvalid)];
      }
      if (DIR == 2) sSrc[E(0)] = sSrc[E(nvalid)];
    }
  }
  // ---- epilogue: face L and the last cell (same thread that wrote the carry)
  if (valid && c == 0) {
    Real qL[5], qR[5], F[5], Fl[5];
#pragma unroll
    for (int v = 0; v < 5; v++) {
      qL[v] = sER[v][E(0)];
      qR[v] = periodic ? sEL0[v][w] : qL[v];
      Fl[v] = sF[v][E(0)];
    }
    if (xhi) {  // a slab bordering another above: the left edge of that slab's first cell
      auto hiSten = [&](int v, int m) -> Real {
        const int p = L - HS + m;
        return p >= L ? XH(1, v, p - L) : ringAt(v, p);
      };
      Real hL[5], hR[5], hs_;
      P::template recon<ORD, DIR>(hiSten, kline, A, hL, hR, hs_, -1L);
#pragma unroll
      for (int v = 0; v < 5; v++) qR[v] = hL[v];
    }
    P::template flux<DIR, NG>(qL, qR, DIR == 2 ? L : kline, A, F);
    if constexpr (PolicyFaceRec<P>::value) P::template face_rec<ORD, DIR>(A, fb + L * fsd, DIR == 2 ? L : kline, qL, qR, F);
    typename P::Aux aux;
    if (A.mode == MODE_APPLY) P::load_aux(A, lb + (L - 1) * sd, sv, aux);
    finish(L - 1, Fl, F, DIR == 2 ? sSrc[E(0)] : Real(0), aux);
  }
  if constexpr (TMA) {  // every issued phase has completed (or been given up on, flagged)
    __syncthreads();
    if (tid == 0) {
      // after a give-up, a last bounded wait so that no box is still landing in this
      // CTA's shared memory when the tile ends
      if (sAbort && phase > 0) (void)mbar_wait(&mbar, (phase - 1) & 1u);
      mbar_inval(&mbar);
    }
  }
}

// TMA: the policy's single-grid TMA path; its tensor map lives in the (grid-constant)
// kernel parameter, the only place besides global memory a TMA copy may read it from.
// CTAs per SM the register budget must allow: the policy's figure, or for the x-slab
// sweeps of ord 5 at least AWFL_SLAB_MINB_ORD5 (4: the FP32 slab sweep drops from 142 to
// 112 registers, no spills, and its x split of a 128x256x128 slab from 0.442 to 0.408 ms;
// the same bound on the single-grid FP32 sweeps made them slower)
#ifndef AWFL_SLAB_MINB_ORD5
#define AWFL_SLAB_MINB_ORD5 4
#endif
template <class P, int ORD, bool SLAB> constexpr int sweep_min_blocks() {
  return (SLAB && ORD == 5 && AWFL_SLAB_MINB_ORD5 > P::min_blocks(ORD)) ? AWFL_SLAB_MINB_ORD5 : P::min_blocks(ORD);
}

template <class P, int ORD, int DIR, int C, int W, bool TMA, bool SLAB = false>
__global__ void __launch_bounds__(C *W, (sweep_min_blocks<P, ORD, SLAB>())) sweep_kernel(const __grid_constant__ typename P::Args A) {
  if constexpr (TMA) sweep_tile<P, ORD, DIR, C, W, true, SLAB>(A, blockIdx.x, blockIdx.y, P::tma_map(A));
  else sweep_tile<P, ORD, DIR, C, W, false, SLAB>(A, blockIdx.x, blockIdx.y);
}

template <int ORD, int DIR> struct SweepShape;
template <> struct SweepShape<5, 0> { static constexpr int C = 32, W = 4; };
template <> struct SweepShape<5, 1> { static constexpr int C = 4, W = 32; };
template <> struct SweepShape<5, 2> { static constexpr int C = 4, W = 32; };
template <> struct SweepShape<9, 0> { static constexpr int C = 32, W = 2; };
template <> struct SweepShape<9, 1> { static constexpr int C = 8, W = 16; };
template <> struct SweepShape<9, 2> { static constexpr int C = 8, W = 16; };

// Shape of a policy's single-grid sweep: SweepShape unless the policy specialises it
// (measured per form at 256x256x128).
template <class P, int ORD, int DIR> struct PolicyShape : SweepShape<ORD, DIR> {};

// Policies with wider elements (P::kWdiv > 1) use fewer lines per CTA to stay within the
// 48 KB of static shared memory.
template <class P, int ORD, int DIR, int C = PolicyShape<P, ORD, DIR>::C,
          int W = (PolicyShape<P, ORD, DIR>::W / P::kWdiv > 0 ? PolicyShape<P, ORD, DIR>::W / P::kWdiv : 1)>
cudaError_t launch_sweep_t(const typename P::Args &A, cudaStream_t st) {
  dim3 block(DIR == 0 ? C : W, DIR == 0 ? W : C);
  dim3 grid;
  if (DIR == 0) grid = dim3((A.ny + W - 1) / W, A.nz);
  else if (DIR == 1) grid = dim3((A.nx + W - 1) / W, A.nz);
  else grid = dim3((A.nx + W - 1) / W, A.ny);
  // the x split of a slab with neighbouring slabs' columns: the SLAB instantiation
  if constexpr (DIR == 0 && P::kSlab) {
    if (A.xh[0] != nullptr || A.xh[1] != nullptr) {
      if constexpr (P::kTmaRing) {
        typename P::Args a = A;
        if (P::prepare_tma(a, ORD, DIR, C, W)) {
          sweep_kernel<P, ORD, DIR, C, W, true, true><<<grid, block, 0, st>>>(a);
          return cudaGetLastError();
        }
      }
      sweep_kernel<P, ORD, DIR, C, W, false, true><<<grid, block, 0, st>>>(A);
      return cudaGetLastError();
    }
  }
  if constexpr (P::kTmaRing) {
    // the policy encodes this launch's tensor map (box = one chunk of one variable); a
    // layout TMA cannot address (alignment) leaves tma off and the cp.async path runs
    typename P::Args a = A;
    if (P::prepare_tma(a, ORD, DIR, C, W)) {
      sweep_kernel<P, ORD, DIR, C, W, true><<<grid, block, 0, st>>>(a);
      return cudaGetLastError();
    }
  }
  sweep_kernel<P, ORD, DIR, C, W, false><<<grid, block, 0, st>>>(A);
  return cudaGetLastError();
}

template <class P>
cudaError_t launch_sweep_any(int ord, int dir, const typename P::Args &A, cudaStream_t st) {
  if (ord == 5) {
    if (dir == 0) return launch_sweep_t<P, 5, 0>(A, st);
    if (dir == 1) return launch_sweep_t<P, 5, 1>(A, st);
    return launch_sweep_t<P, 5, 2>(A, st);
  }
  if (dir == 0) return launch_sweep_t<P, 9, 0>(A, st);
  if (dir == 1) return launch_sweep_t<P, 9, 1>(A, st);
  return launch_sweep_t<P, 9, 2>(A, st);
}

}  // namespace awfl
