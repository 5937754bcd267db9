// Blake3 Merkle trees on the device, byte-compatible with the reference's
// `MerkleTreeProver` (utils/src/merkle.rs:49-85 over rs_merkle 1.5.0): a leaf is
// blake3(serialized field elements), a parent is blake3(left || right).  Nodes are stored as
// 8 little-endian u32 words, all layers in one buffer: layer 0 (leaves) first, then each parent
// layer, the root last.  Every tree on this path has a power-of-two leaf count.
#include "blake3.cuh"
#include "kernels.cuh"

namespace lgs {

// Leaf p is the `words` consecutive u64 starting at data[p * words] (leaf-major layouts).
__global__ void leaf_hash_contig_kernel(const u64* __restrict__ data, unsigned words,
                                        size_t nleaves, u32* __restrict__ out) {
  size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nleaves) return;
  const u64* src = data + p * words;
  u32 cv[8];
  b3_init(cv);
  const unsigned len = words * 8;
  const unsigned nblocks = (len + 63) / 64;
  for (unsigned b = 0; b < nblocks; ++b) {
    u32 blk[16];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      unsigned w = b * 8 + q;
      u64 v = w < words ? src[w] : 0;
      blk[2 * q] = (u32)v;
      blk[2 * q + 1] = (u32)(v >> 32);
    }
    unsigned bl = len - b * 64 < 64 ? len - b * 64 : 64;
    u32 flags = (b == 0 ? B3_CHUNK_START : 0) | (b + 1 == nblocks ? (B3_CHUNK_END | B3_ROOT) : 0);
    b3_compress(cv, blk, bl, flags);
  }
#pragma unroll
  for (int q = 0; q < 8; ++q) out[p * 8 + q] = cv[q];
}

// Turns 2^q consecutive nodes (starting at block index `blk` of a layer at in_off with in_count
// nodes) into the q layers above them.  Needs 2^(q-1) <= blockDim.x, sh >= 2^(q-1) nodes.
__device__ void subtree_reduce(u32* __restrict__ nodes, size_t in_off, size_t in_count, unsigned q,
                               size_t blk, u32* sh) {
  const unsigned half0 = 1u << (q - 1);
  size_t layer_off = in_off, layer_count = in_count;
  unsigned cnt = half0;
  size_t local_base = blk << q;  // index of this CTA's first node within the current layer
  for (unsigned i = threadIdx.x; i < cnt; i += blockDim.x) {
    const u32* l = nodes + (layer_off + local_base + 2 * i) * 8;
    u32 lw[8], rw[8], o[8];
#pragma unroll
    for (int w = 0; w < 8; ++w) lw[w] = l[w], rw[w] = l[8 + w];
    b3_parent(lw, rw, o);
#pragma unroll
    for (int w = 0; w < 8; ++w) sh[i * 8 + w] = o[w];
  }
  __syncthreads();
  for (unsigned lev = 1; lev <= q; ++lev) {
    size_t next_off = layer_off + layer_count;
    size_t next_base = local_base >> 1;
    for (unsigned i = threadIdx.x; i < cnt * 8; i += blockDim.x)
      nodes[(next_off + next_base) * 8 + i] = sh[i];
    if (lev == q) break;
    __syncthreads();
    unsigned ncnt = cnt >> 1;
    u32 o[8];
    bool act = threadIdx.x < ncnt;
    if (act) {
      u32 lw[8], rw[8];
#pragma unroll
      for (int w = 0; w < 8; ++w) lw[w] = sh[threadIdx.x * 16 + w], rw[w] = sh[threadIdx.x * 16 + 8 + w];
      b3_parent(lw, rw, o);
    }
    __syncthreads();
    if (act)
#pragma unroll
      for (int w = 0; w < 8; ++w) sh[threadIdx.x * 8 + w] = o[w];
    __syncthreads();
    layer_off = next_off;
    layer_count >>= 1;
    local_base = next_base;
    cnt = ncnt;
  }
}

__global__ void tree_reduce_kernel(u32* __restrict__ nodes, size_t in_off, size_t in_count,
                                   unsigned q) {
  extern __shared__ u32 sh[];  // 2^(q-1) nodes x 8 words
  subtree_reduce(nodes, in_off, in_count, q, blockIdx.x, sh);
}

struct TreeJob {
  u32* nodes;
  size_t in_off, in_count;
  unsigned q, first_cta;
};
struct TreeJobs {
  TreeJob j[16];
  unsigned n;
};
__global__ void tree_reduce_many_kernel(const TreeJobs jobs) {
  __shared__ u32 sh[256 * 8];
  unsigned t = 0;
  while (t + 1 < jobs.n && blockIdx.x >= jobs.j[t + 1].first_cta) ++t;
  const TreeJob& jb = jobs.j[t];
  subtree_reduce(jb.nodes, jb.in_off, jb.in_count, jb.q, blockIdx.x - jb.first_cta, sh);
}

struct LeafJobs {
  const u64* data[16];
  u32* nodes[16];
  size_t first[17];  // prefix sums of leaf counts
  unsigned n, words;
};
__global__ void leaf_hash_many_kernel(const LeafJobs jobs) {
  const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= jobs.first[jobs.n]) return;
  unsigned t = 0;
  while (g >= jobs.first[t + 1]) ++t;
  const size_t p = g - jobs.first[t];
  const u64* src = jobs.data[t] + p * jobs.words;
  const unsigned len = jobs.words * 8, nblocks = (len + 63) / 64;
  u32 cv[8];
  b3_init(cv);
  for (unsigned b = 0; b < nblocks; ++b) {
    u32 blk[16];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const unsigned w = b * 8 + q;
      const u64 v = w < jobs.words ? src[w] : 0;
      blk[2 * q] = (u32)v;
      blk[2 * q + 1] = (u32)(v >> 32);
    }
    const unsigned bl = len - b * 64 < 64 ? len - b * 64 : 64;
    const u32 flags = (b == 0 ? B3_CHUNK_START : 0) | (b + 1 == nblocks ? (B3_CHUNK_END | B3_ROOT) : 0);
    b3_compress(cv, blk, bl, flags);
  }
#pragma unroll
  for (int q = 0; q < 8; ++q) jobs.nodes[t][p * 8 + q] = cv[q];
}

size_t merkle_node_count(size_t nleaves) { return 2 * nleaves - 1; }
size_t merkle_layer_offset(size_t nleaves, unsigned layer) {
  size_t off = 0, cnt = nleaves;
  for (unsigned l = 0; l < layer; ++l) {
    off += cnt;
    cnt >>= 1;
  }
  return off;
}

// Build parents for a tree whose leaf hashes are already in nodes[0 .. nleaves).
void merkle_build_from_leaves(u32* nodes, size_t nleaves, cudaStream_t st) {
  if (nleaves & (nleaves - 1)) throw ShapeError("merkle: leaf count must be a power of two");
  size_t off = 0, count = nleaves;
  while (count > 1) {
    unsigned logc = ilog2(count);
    unsigned q = logc < 9 ? logc : 9;
    unsigned half0 = 1u << (q - 1);
    unsigned threads = half0 < 256 ? (half0 < 32 ? 32 : half0) : 256;
    size_t grid = count >> q;
    tree_reduce_kernel<<<(unsigned)grid, threads, half0 * 32, st>>>(nodes, off, count, q);
    LGS_LAUNCH_CHECK();
    // advance q layers
    for (unsigned t = 0; t < q; ++t) {
      off += count;
      count >>= 1;
    }
  }
}

void merkle_leaves_contig(const u64* data, unsigned words, size_t nleaves, u32* nodes,
                          cudaStream_t st) {
  if (words * 8 > 1024) throw ShapeError("merkle: leaf larger than one blake3 chunk");
  leaf_hash_contig_kernel<<<cdiv(nleaves, 128), 128, 0, st>>>(data, words, nleaves, nodes);
  LGS_LAUNCH_CHECK();
}

void merkle_build_many(u32* const* nodes, const size_t* nleaves, unsigned ntrees,
                       cudaStream_t st) {
  if (ntrees > 16) throw ShapeError("merkle: at most 16 trees per batch");
  size_t off[16], count[16];
  for (unsigned t = 0; t < ntrees; ++t) {
    if (nleaves[t] == 0 || (nleaves[t] & (nleaves[t] - 1)))
      throw ShapeError("merkle: leaf count must be a power of two");
    off[t] = 0;
    count[t] = nleaves[t];
  }
  while (true) {
    TreeJobs jobs;
    jobs.n = 0;
    unsigned ctas = 0;
    for (unsigned t = 0; t < ntrees; ++t) {
      if (count[t] <= 1) continue;
      const unsigned logc = ilog2(count[t]);
      const unsigned q = logc < 9 ? logc : 9;
      TreeJob& jb = jobs.j[jobs.n++];
      jb.nodes = nodes[t];
      jb.in_off = off[t];
      jb.in_count = count[t];
      jb.q = q;
      jb.first_cta = ctas;
      ctas += (unsigned)(count[t] >> q);
      for (unsigned i = 0; i < q; ++i) {
        off[t] += count[t];
        count[t] >>= 1;
      }
    }
    if (!jobs.n) break;
    tree_reduce_many_kernel<<<ctas, 256, 0, st>>>(jobs);
    LGS_LAUNCH_CHECK();
  }
}

void merkle_leaves_many(const u64* const* data, unsigned words, u32* const* nodes,
                        const size_t* nleaves, unsigned ntrees, cudaStream_t st) {
  if (ntrees > 16 || ntrees == 0) throw ShapeError("merkle: 1 to 16 trees per batch");
  if (words * 8 > 1024) throw ShapeError("merkle: leaf larger than one blake3 chunk");
  LeafJobs jobs;
  jobs.n = ntrees;
  jobs.words = words;
  jobs.first[0] = 0;
  for (unsigned t = 0; t < ntrees; ++t) {
    jobs.data[t] = data[t];
    jobs.nodes[t] = nodes[t];
    jobs.first[t + 1] = jobs.first[t] + nleaves[t];
  }
  leaf_hash_many_kernel<<<cdiv(jobs.first[ntrees], 128), 128, 0, st>>>(jobs);
  LGS_LAUNCH_CHECK();
}

// dst[i] = src[idx[i]] for `count` items of `words` u64 each.
__global__ void gather_kernel(const u64* __restrict__ src, const uint64_t* __restrict__ idx,
                              size_t count, unsigned words, u64* __restrict__ dst) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count * words) return;
  size_t i = t / words, w = t % words;
  dst[t] = src[idx[i] * words + w];
}
void gather_u64(const u64* src, const uint64_t* idx, size_t count, unsigned words, u64* dst,
                cudaStream_t st) {
  if (!count) return;
  gather_kernel<<<cdiv(count * words, 256), 256, 0, st>>>(src, idx, count, words, dst);
  LGS_LAUNCH_CHECK();
}

}  // namespace lgs
