// C ABI: host tree serialisation (sbh_host_tree_save / sbh_host_tree_load).
//
// A file holds one HostTree: a fixed header, every array of the tree as
// (element count, raw little-endian elements) in a fixed order, and an FNV-1a
// 64-bit checksum of everything before it.  Loading checks the header, every
// array's length against the header's sizes, the checksum, and the tree's
// structure (point ranges, child indices, parents, levels), so that a damaged
// or foreign file is refused instead of reaching a device walk.
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "internal.h"

namespace {

constexpr char kMagic[8] = {'S', 'B', 'H', 'T', 'R', 'E', 'E', '1'};
constexpr uint32_t kVersion = 1;

struct Header {
  char magic[8];
  uint32_t version;
  int32_t dim, dsl, leaf_size, max_depth, depth;
  int64_t n, nn;
  float alpha;
  int32_t pad;
};

struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void add(const void* p, size_t bytes) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < bytes; i++) {
      h ^= c[i];
      h *= 1099511628211ull;
    }
  }
};

struct Writer {
  FILE* f;
  Fnv sum;
  bool ok = true;
  void raw(const void* p, size_t bytes) {
    if (!ok || bytes == 0) return;
    ok = std::fwrite(p, 1, bytes, f) == bytes;
    sum.add(p, bytes);
  }
  template <typename T>
  void array(const std::vector<T>& v) {
    const uint64_t count = v.size();
    raw(&count, sizeof(count));
    raw(v.data(), v.size() * sizeof(T));
  }
};

struct Reader {
  FILE* f;
  Fnv sum;
  bool ok = true;
  void raw(void* p, size_t bytes) {
    if (!ok || bytes == 0) return;
    ok = std::fread(p, 1, bytes, f) == bytes;
    if (ok) sum.add(p, bytes);
  }
  // Reads an array that must hold exactly `expect` elements.
  template <typename T>
  void array(std::vector<T>& v, uint64_t expect) {
    uint64_t count = 0;
    raw(&count, sizeof(count));
    if (!ok || count != expect) {
      ok = false;
      return;
    }
    v.resize(static_cast<size_t>(count));
    raw(v.data(), v.size() * sizeof(T));
  }
};

// Structural checks of a loaded tree: everything a device walk indexes with.
std::string check_structure(const sbh::HostTree& t) {
  if (t.dim != 2 && t.dim != 3) return "dimension must be 2 or 3";
  if (t.dsl < 1 || t.dsl > 3) return "dim_split_log must be 1..3";
  if (t.ds != (1 << t.dsl) || t.bf != (1 << (t.dim * t.dsl)) ||
      t.mw != (t.bf >= 64 ? t.bf / 64 : 1))
    return "inconsistent branching";
  if (t.n < 0 || t.n > (int64_t)INT32_MAX || t.nn < 1 || t.nn > (int64_t)INT32_MAX)
    return "point or node count out of range";
  if (t.level_begin.empty() || t.level_begin.front() != 0 || t.level_begin.back() != t.nn)
    return "bad level table";
  for (size_t l = 1; l < t.level_begin.size(); l++)
    if (t.level_begin[l] <= t.level_begin[l - 1]) return "bad level table";
  if (t.start[0] != 0 || t.end[0] != t.n) return "root must hold every point";
  for (int64_t v = 0; v < t.nn; v++) {
    if (t.start[v] < 0 || t.start[v] > t.end[v] || t.end[v] > t.n) return "bad point range";
    if (v > 0 && (t.parent[v] < 0 || t.parent[v] >= v)) return "bad parent";
    if (t.node_depth[v] < 0 || t.node_depth[v] > t.depth) return "bad depth";
    if (!t.leaf[v]) {
      const int64_t c = t.first_child[v], k = t.nch[v];
      if (k < 1 || k > t.bf || c <= v || c + k > t.nn) return "bad child range";
      int bits = 0;
      for (int w = 0; w < t.mw; w++) bits += __builtin_popcountll(t.mask[v * t.mw + w]);
      if (bits != k) return "child mask does not match the child count";
      for (int64_t u = c; u < c + k; u++)
        if (t.parent[u] != v || t.node_depth[u] != t.node_depth[v] + 1)
          return "child does not point back to its parent";
      if (t.start[c] != t.start[v] || t.end[c + k - 1] != t.end[v]) return "children do not tile";
      for (int64_t u = c + 1; u < c + k; u++)
        if (t.start[u] != t.end[u - 1]) return "children do not tile";
    }
  }
  return "";
}

}  // namespace

SBH_API int sbh_host_tree_save(const sbh_host_tree* tree, const char* path) {
  if (!tree || !path) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null tree or path");
  const sbh::HostTree& t = tree->t;
  FILE* f = std::fopen(path, "wb");
  if (!f) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
  Header h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kMagic, sizeof(kMagic));
  h.version = kVersion;
  h.dim = t.dim;
  h.dsl = t.dsl;
  h.leaf_size = t.leaf_size;
  h.max_depth = t.max_depth;
  h.depth = t.depth;
  h.n = t.n;
  h.nn = t.nn;
  h.alpha = t.alpha;
  Writer w{f, Fnv(), true};
  w.raw(&h, sizeof(h));
  w.array(t.pos); w.array(t.nrm); w.array(t.mass);
  w.array(t.start); w.array(t.end); w.array(t.parent); w.array(t.first_child);
  w.array(t.node_depth); w.array(t.nch); w.array(t.leaf); w.array(t.mask);
  w.array(t.bmin); w.array(t.bmax); w.array(t.diam);
  w.array(t.amass); w.array(t.apos); w.array(t.anrm); w.array(t.aalpha);
  w.array(t.level_begin);
  const uint64_t sum = w.sum.h;
  bool ok = w.ok && std::fwrite(&sum, 1, sizeof(sum), f) == sizeof(sum);
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
  return sbh::ok();
}

SBH_API int sbh_host_tree_load(const char* path, sbh_host_tree** out) {
  if (!path || !out) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, "null path or out");
  *out = nullptr;
  FILE* f = std::fopen(path, "rb");
  if (!f) return sbh::fail(SBH_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
  sbh_host_tree* h = new (std::nothrow) sbh_host_tree();
  if (!h) {
    std::fclose(f);
    return sbh::fail(SBH_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
  std::string err;
  try {
    Reader r{f, Fnv(), true};
    Header hd;
    r.raw(&hd, sizeof(hd));
    if (!r.ok || std::memcmp(hd.magic, kMagic, sizeof(kMagic)) != 0)
      err = "not a tree file";
    else if (hd.version != kVersion)
      err = "unsupported tree file version";
    else if ((hd.dim != 2 && hd.dim != 3) || hd.dsl < 1 || hd.dsl > 3 || hd.n < 0 ||
             hd.n > (int64_t)INT32_MAX || hd.nn < 1 || hd.nn > (int64_t)INT32_MAX || hd.depth < 0)
      err = "tree file header out of range";
    if (err.empty()) {
      sbh::HostTree& t = h->t;
      t.dim = hd.dim;
      t.dsl = hd.dsl;
      t.ds = 1 << hd.dsl;
      t.bf = 1 << (hd.dim * hd.dsl);
      t.mw = t.bf >= 64 ? t.bf / 64 : 1;
      t.leaf_size = hd.leaf_size;
      t.max_depth = hd.max_depth;
      t.depth = hd.depth;
      t.n = hd.n;
      t.nn = hd.nn;
      t.alpha = hd.alpha;
      const uint64_t n = hd.n, nn = hd.nn, d = hd.dim;
      r.array(t.pos, n * d); r.array(t.nrm, n * d); r.array(t.mass, n);
      r.array(t.start, nn); r.array(t.end, nn); r.array(t.parent, nn); r.array(t.first_child, nn);
      r.array(t.node_depth, nn); r.array(t.nch, nn); r.array(t.leaf, nn);
      r.array(t.mask, nn * t.mw);
      r.array(t.bmin, nn * d); r.array(t.bmax, nn * d); r.array(t.diam, nn);
      r.array(t.amass, nn); r.array(t.apos, nn * d); r.array(t.anrm, nn * d);
      r.array(t.aalpha, nn);
      r.array(t.level_begin, (uint64_t)hd.depth + 2);
      const uint64_t expect = r.sum.h;
      uint64_t sum = 0;
      if (!r.ok || std::fread(&sum, 1, sizeof(sum), f) != sizeof(sum))
        err = "tree file is truncated or its arrays have the wrong sizes";
      else if (sum != expect)
        err = "tree file checksum mismatch";
      else
        err = check_structure(t);
    }
  } catch (const std::bad_alloc&) {
    err = "out of memory reading the tree file";
  }
  std::fclose(f);
  if (!err.empty()) {
    delete h;
    return sbh::fail(SBH_ERR_INVALID_ARGUMENT, err);
  }
  *out = h;
  return sbh::ok();
}
