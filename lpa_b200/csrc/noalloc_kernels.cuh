// Kernels of lpa_iterate_noalloc (host side: noalloc.cu).  Included at the
// end of lp_kernels.cu so they share its device functions.
#pragma once

// ---------------------------------------------------------------------------
// Two-pass iteration without allocations (host side: noalloc.cu).
// ---------------------------------------------------------------------------
__global__ void k_na_degrees(NoAllocArgs a) {
  const DevGraph &g = a.g;
  uint32_t my_max = 0;
  for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < g.n; p += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t d = 0;
    if (g.vertices[p] >= g.n) {
      set_error(a.err, kErrBadStream);
    } else if (p < g.n_c) {
      const uint64_t b = g.offsets[p], e = g.offsets[p + 1];
      if (e < b || e > a.total_bits) {  // out-of-order or out-of-stream offsets: never read there
        set_error(a.err, kErrBadStream);
      } else {
        const int64_t c = walk_vertex_buf(g.words, b, e, g.vertices[p], g.n, [](uint32_t) {});
        if (c < 0 || c > int64_t(0xFFFFFFFFll)) set_error(a.err, kErrBadStream);
        else d = uint32_t(c);
      }
    } else {
      const uint32_t b = g.small_off[p - g.n_c], e = g.small_off[p - g.n_c + 1];
      if (e < b || e > a.small_arcs) {
        set_error(a.err, kErrBadStream);
      } else {
        d = e - b;
        for (uint32_t k = b; k < e; k++)
          if (g.small_nbr[k] >= g.n) {
            set_error(a.err, kErrBadStream);
            d = 0;
            break;
          }
      }
    }
    a.deg[p] = d;
    my_max = d > my_max ? d : my_max;
  }
  if (my_max) atomicMax(a.stats + 1, (unsigned long long)my_max);
}

// Exclusive scan of the compressed positions' degrees (one block).
__global__ void k_na_scan(NoAllocArgs a) {
  __shared__ unsigned long long part[1024];
  const uint64_t n_c = a.g.n_c;
  const uint32_t t = threadIdx.x, T = blockDim.x;
  const uint64_t per = (n_c + T - 1) / T;
  const uint64_t b = min(n_c, per * t), e = min(n_c, b + per);
  unsigned long long s = 0;
  for (uint64_t p = b; p < e; p++) s += a.deg[p];
  part[t] = s;
  __syncthreads();
  if (t == 0) {
    unsigned long long acc = 0;
    for (uint32_t i = 0; i < T; i++) {
      const unsigned long long v = part[i];
      part[i] = acc;
      acc += v;
    }
    a.arc_off[n_c] = acc;
    a.stats[2] = acc;
  }
  __syncthreads();
  unsigned long long acc = part[t];
  for (uint64_t p = b; p < e; p++) {
    a.arc_off[p] = acc;
    acc += a.deg[p];
  }
}

// Pass 1: warps decode 32 compressed positions at a time into ids.
__global__ void __launch_bounds__(kThreads) k_na_decode(NoAllocArgs a) {
  const DevGraph &g = a.g;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t chunks = (g.n_c + 31) / 32;
  for (uint64_t ch = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) / 32; ch < chunks;
       ch += uint64_t(gridDim.x) * blockDim.x / 32) {
    const uint32_t p0 = uint32_t(ch * 32);
    const uint32_t p = p0 + lane;
    const bool valid = p < g.n_c;
    const uint32_t node = valid ? g.vertices[p] : 0u;
    const uint32_t d = valid ? a.deg[p] : 0u;
    const uint64_t o0 = a.arc_off[p0];
    const uint32_t base = valid ? uint32_t(a.arc_off[p] - o0) : 0u;
    if (!warp_decode_batch(g, a.ids + o0, valid, p, node, d, base, lane) && lane == 0) set_error(a.err, kErrBadStream);
  }
}

// Pass 2: warps count 32 positions at a time from ids (compressed positions)
// or the small CSR, one vertex per round (degrees <= kV1MaxDeg, exact).
__global__ void __launch_bounds__(kThreads, 2) k_na_count(NoAllocArgs a) {
  extern __shared__ uint32_t smem[];
  __shared__ IterArgs ia;
  const uint32_t t = threadIdx.x, warp = t >> 5;
  uint32_t *stage = smem;
  uint32_t *tab = smem + kStage;
  for (uint32_t i = t; i < 2 * kTableSlots; i += kThreads) tab[i] = 0u;
  if (t == 0) {
    ia = IterArgs{};
    ia.g = a.g;
    ia.err = a.err;
    ia.scratch = a.ids;
    ia.arc_off = a.arc_off;
    ia.cms_thr = a.cms_thr;
  }
  __syncthreads();
  Ctx c;
  c.it = 0;
  c.lab_in = a.lab_in;
  c.lab_out = a.lab_out;
  c.changed = a.stats;
  c.coherent = false;
  unsigned long long *wslots = reinterpret_cast<unsigned long long *>(tab) + warp * kWarpSlots;
  uint32_t *wstage = stage + warp * kWarpStage;
  uint32_t wepoch = 0;
  unsigned long long changed = 0;
  const DevGraph &g = a.g;
  const uint64_t cchunks = (g.n_c + 31) / 32, schunks = (g.n - g.n_c + 31) / 32;
  for (uint64_t ch = (blockIdx.x * uint64_t(blockDim.x) + t) / 32; ch < cchunks + schunks;
       ch += uint64_t(gridDim.x) * blockDim.x / 32) {
    uint32_t p0, p1;
    if (ch < cchunks) {
      p0 = uint32_t(ch * 32);
      p1 = uint32_t(g.n_c < uint64_t(p0) + 32ull ? g.n_c : uint64_t(p0) + 32ull);
    } else {
      p0 = uint32_t(g.n_c + (ch - cchunks) * 32);
      p1 = uint32_t(g.n < uint64_t(p0) + 32ull ? g.n : uint64_t(p0) + 32ull);
    }
    light_chunk(ia, c, wstage, wslots, wepoch, 0, p0, p1, kVarTwoPass, changed);
  }
  flush_changed(c.changed, changed);
}

