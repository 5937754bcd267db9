// ORACLE (test infrastructure only): the Blake3 Merkle tree of utils/src/merkle.rs:5-117,
// restated over the behaviour of rs_merkle 1.5.0 (Cargo.lock:559) that the reference uses:
//   * `MerkleTree::from_leaves(leaf_hashes)` (utils/src/merkle.rs:59-66): layer 0 holds the leaf
//     hashes; a parent is `Blake32::hash(left || right)` (rs_merkle's default
//     `concat_and_hash`); an unpaired last node is promoted unchanged.  All trees on this path
//     have a power-of-two leaf count, so no node is ever promoted.
//   * `proof(indices).to_bytes()` (utils/src/merkle.rs:76-78): for each layer from the leaves up,
//     the siblings of the current index set that are not themselves in the set, in increasing
//     index order; the set then moves to the (deduplicated) parents.  The bytes are those
//     32-byte hashes concatenated (rs_merkle's DirectHashesOrder).
//   * `MerkleProof::verify` (utils/src/merkle.rs:89-103): rebuild the root from the leaf hashes
//     and the proof hashes with the same layer walk; accept iff it equals the root.
// This byte layout is the one rs_merkle documents; no reference test pins it.
#pragma once
#include <algorithm>
#include <array>
#include <cstdint>
#include <map>
#include <vector>

#include "blake3_ref.hpp"
#include "gl.hpp"
#include "par.hpp"

namespace orc {

using Hash = std::array<uint8_t, 32>;

inline Hash hash_bytes(const uint8_t* p, size_t n) {
  Hash h;
  Blake3::hash(p, n, h.data());
  return h;
}
inline Hash hash_pair(const Hash& l, const Hash& r) {
  uint8_t buf[64];
  std::copy(l.begin(), l.end(), buf);
  std::copy(r.begin(), r.end(), buf + 32);
  return hash_bytes(buf, 64);
}

inline size_t tree_depth(size_t leaves) {
  size_t d = 0;
  while ((size_t(1) << d) < leaves) ++d;
  return d;
}

// Per layer: the proof-node indices for a sorted, deduplicated leaf index set.
inline std::vector<std::vector<size_t>> proof_indices_by_layers(std::vector<size_t> cur,
                                                                size_t leaves) {
  std::vector<std::vector<size_t>> out;
  size_t depth = tree_depth(leaves);
  size_t layer_len = leaves;
  for (size_t layer = 0; layer < depth; ++layer) {
    std::vector<size_t> sib;
    for (size_t i : cur) {
      size_t s = i ^ 1;
      if (s >= layer_len) continue;  // unpaired last node (never hit for 2^k leaves)
      if (!std::binary_search(cur.begin(), cur.end(), s)) sib.push_back(s);
    }
    out.push_back(sib);
    std::vector<size_t> parents;
    for (size_t i : cur)
      if (parents.empty() || parents.back() != i / 2) parents.push_back(i / 2);
    cur.swap(parents);
    layer_len = (layer_len + 1) / 2;
  }
  return out;
}

struct MerkleTree {
  std::vector<std::vector<Hash>> layers;  // layers[0] = leaf hashes, last = {root}
  size_t leaves() const { return layers[0].size(); }
  static MerkleTree from_leaf_hashes(std::vector<Hash> lh) {
    MerkleTree t;
    t.layers.push_back(std::move(lh));
    while (t.layers.back().size() > 1) {
      const auto& cur = t.layers.back();
      std::vector<Hash> next((cur.size() + 1) / 2);
      parallel_ranges(next.size(), [&](size_t lo, size_t hi) {
        for (size_t k = lo; k < hi; ++k) {
          size_t i = 2 * k;
          next[k] = i + 1 < cur.size() ? hash_pair(cur[i], cur[i + 1]) : cur[i];
        }
      }, size_t(1) << 12);
      t.layers.push_back(std::move(next));
    }
    return t;
  }
  static MerkleTree from_leaves(const std::vector<std::vector<uint8_t>>& leaves) {
    std::vector<Hash> lh;
    lh.reserve(leaves.size());
    for (auto& l : leaves) lh.push_back(hash_bytes(l.data(), l.size()));
    return from_leaf_hashes(std::move(lh));
  }
  Hash root() const { return layers.back()[0]; }
  // `indices` must be sorted and distinct (every caller on the path passes such a set).
  std::vector<uint8_t> open(const std::vector<size_t>& indices) const {
    auto by_layer = proof_indices_by_layers(indices, leaves());
    std::vector<uint8_t> out;
    for (size_t l = 0; l < by_layer.size(); ++l)
      for (size_t i : by_layer[l]) out.insert(out.end(), layers[l][i].begin(), layers[l][i].end());
    return out;
  }
};

// Rebuild the root from (sorted, distinct) indices, their leaf hashes and the proof bytes.
// Returns false when the proof is malformed (wrong length, missing nodes).
inline bool merkle_root_from_proof(const std::vector<uint8_t>& proof,
                                   const std::vector<size_t>& indices,
                                   const std::vector<Hash>& leaf_hashes, size_t leaves,
                                   Hash* root) {
  if (indices.size() != leaf_hashes.size() || indices.empty()) return false;
  for (size_t i = 0; i < indices.size(); ++i) {
    if (indices[i] >= leaves) return false;
    if (i && indices[i] <= indices[i - 1]) return false;
  }
  if (proof.size() % 32) return false;
  auto by_layer = proof_indices_by_layers(indices, leaves);
  size_t total = 0;
  for (auto& v : by_layer) total += v.size();
  if (total * 32 != proof.size()) return false;
  std::map<size_t, Hash> known;
  for (size_t i = 0; i < indices.size(); ++i) known[indices[i]] = leaf_hashes[i];
  size_t pos = 0, layer_len = leaves;
  for (size_t l = 0; l < by_layer.size(); ++l) {
    for (size_t i : by_layer[l]) {
      Hash h;
      std::copy(proof.begin() + pos, proof.begin() + pos + 32, h.begin());
      pos += 32;
      known[i] = h;
    }
    std::map<size_t, Hash> next;
    for (auto it = known.begin(); it != known.end(); ++it) {
      size_t i = it->first;
      if (i & 1) continue;
      auto r = known.find(i + 1);
      if (r == known.end()) {
        if (i + 1 < layer_len) return false;  // sibling needed but absent
        next[i / 2] = it->second;
      } else {
        next[i / 2] = hash_pair(it->second, r->second);
      }
    }
    for (auto& kv : known)
      if ((kv.first & 1) && !known.count(kv.first - 1)) return false;
    known.swap(next);
    layer_len = (layer_len + 1) / 2;
  }
  if (known.size() != 1 || known.begin()->first != 0) return false;
  *root = known.begin()->second;
  return true;
}

inline bool merkle_verify(const Hash& root, const std::vector<uint8_t>& proof,
                          const std::vector<size_t>& indices,
                          const std::vector<std::vector<uint8_t>>& leaves, size_t leave_number) {
  std::vector<Hash> lh;
  for (auto& l : leaves) lh.push_back(hash_bytes(l.data(), l.size()));
  Hash r;
  if (!merkle_root_from_proof(proof, indices, lh, leave_number, &r)) return false;
  return r == root;
}

// `Serialize::serialize_fields` (utils/src/merkle.rs:24-35): canonical u64 little-endian; an EF
// element as c0 then c1.
inline void ser_u64(std::vector<uint8_t>& out, u64 v) {
  for (int i = 0; i < 8; ++i) out.push_back((uint8_t)(v >> (8 * i)));
}
inline std::vector<uint8_t> serialize_bf(const std::vector<u64>& v) {
  std::vector<uint8_t> out;
  out.reserve(v.size() * 8);
  for (u64 x : v) ser_u64(out, canon(x));
  return out;
}
inline std::vector<uint8_t> serialize_ef(const std::vector<EF>& v) {
  std::vector<uint8_t> out;
  out.reserve(v.size() * 16);
  for (const EF& x : v) {
    ser_u64(out, canon(x.c0));
    ser_u64(out, canon(x.c1));
  }
  return out;
}

}  // namespace orc
