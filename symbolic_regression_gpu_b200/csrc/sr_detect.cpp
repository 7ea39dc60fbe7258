// sr_detect.cpp — common-subtree detection and cache marking.
#include "sr_detect.hpp"

#include <algorithm>
#include <cstring>

#include "sr_program.hpp"

namespace sr {

namespace {
inline uint64_t dbits(double v) {
  uint64_t u;
  std::memcpy(&u, &v, sizeof u);
  return u;
}
// Sign-extending int -> uint64 conversion, as the reference's (uint64_t)token.
inline uint64_t tbits(int32_t t) {
  return static_cast<uint64_t>(static_cast<int64_t>(t));
}
}  // namespace

uint64_t flat_key(const int32_t *tok, const double *val, int len) {
  uint64_t h = kFnvOffset;
  for (int i = 0; i < len; ++i) {
    h ^= tbits(tok[i]);
    h *= kFnvPrime;
    h ^= dbits(val[i]);
    h *= kFnvPrime;
  }
  return h;
}

uint64_t merkle_node(int32_t tok, double val, const uint64_t *child, int nchild) {
  uint64_t h = kFnvOffset;
  h ^= tbits(tok);
  h *= kFnvPrime;
  h ^= dbits(val);
  h *= kFnvPrime;
  for (int k = 0; k < nchild; ++k)
    h = h ^ (child[k] + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2));
  return h;
}

void merkle_hashes(const int32_t *tok, const double *val, int len,
                   int32_t *sizes, uint64_t *hashes) {
  for (int i = len - 1; i >= 0; --i) {
    const int t = tok[i];
    if (t <= 0) {
      sizes[i] = 1;
      hashes[i] = merkle_node(t, val[i], nullptr, 0);
      continue;
    }
    const int arity = (t < 10) ? 2 : 1;
    uint64_t ch[2];
    int nch = 0, size = 1, pos = i + 1;
    for (int k = 0; k < arity && pos < len; ++k) {
      size += sizes[pos];
      ch[nch++] = hashes[pos];
      pos += sizes[pos];
    }
    sizes[i] = size;
    hashes[i] = merkle_node(t, val[i], ch, nch);
  }
}

namespace {
struct Candidate {
  uint64_t hash;
  int32_t expr, pos, size;
};
}  // namespace

void detect_common_subtrees(int E, const int32_t *tok, const double *val,
                            const int64_t *off, int min_size, int min_freq,
                            int threads, Detection &out) {
  out = Detection{};
  out.total_tokens = E > 0 ? off[E] - off[0] : 0;
  if (E <= 0) return;

  // Step 1: per-expression reverse pass -> candidates (parallel over
  // expressions, merged in expression order).
  const int nt = std::max(1, threads);
  std::vector<std::vector<Candidate>> part(static_cast<size_t>(nt));
  parallel_for(nt, nt, [&](int64_t b, int64_t e) {
    std::vector<int32_t> sizes;
    std::vector<uint64_t> hashes;
    for (int64_t c = b; c < e; ++c) {
      auto &dst = part[static_cast<size_t>(c)];
      const int64_t x0 = E * c / nt, x1 = E * (c + 1) / nt;
      for (int64_t x = x0; x < x1; ++x) {
        const int len = static_cast<int>(off[x + 1] - off[x]);
        sizes.resize(static_cast<size_t>(len));
        hashes.resize(static_cast<size_t>(len));
        merkle_hashes(tok + off[x], val + off[x], len, sizes.data(), hashes.data());
        for (int i = len - 1; i >= 0; --i)
          if (sizes[i] >= min_size)
            dst.push_back(Candidate{hashes[i], static_cast<int32_t>(x), i, sizes[i]});
      }
    }
  });
  std::vector<Candidate> cand;
  {
    size_t total = 0;
    for (auto &p : part) total += p.size();
    cand.reserve(total);
    for (auto &p : part) cand.insert(cand.end(), p.begin(), p.end());
  }
  std::sort(cand.begin(), cand.end(), [](const Candidate &a, const Candidate &b) {
    if (a.hash != b.hash) return a.hash < b.hash;
    if (a.expr != b.expr) return a.expr < b.expr;
    return a.pos < b.pos;
  });

  // Step 2: group equal hashes, verify against the first member.
  struct VGroup {
    int32_t size;
    size_t first;                  // index into `members`
    int32_t count;
  };
  std::vector<VGroup> groups;
  std::vector<Candidate> members;
  for (size_t i = 0; i < cand.size();) {
    size_t j = i + 1;
    while (j < cand.size() && cand[j].hash == cand[i].hash) ++j;
    if (static_cast<int>(j - i) >= min_freq) {
      const Candidate &ref = cand[i];
      const int32_t *rt = tok + off[ref.expr] + ref.pos;
      const double *rv = val + off[ref.expr] + ref.pos;
      const size_t start = members.size();
      for (size_t k = i; k < j; ++k) {
        const Candidate &c = cand[k];
        if (c.size != ref.size) continue;
        const int32_t *ct = tok + off[c.expr] + c.pos;
        const double *cv = val + off[c.expr] + c.pos;
        bool same = true;
        for (int q = 0; q < ref.size && same; ++q)
          same = (rt[q] == ct[q]) && (rv[q] == cv[q]);
        if (same) members.push_back(c);
      }
      const int32_t cnt = static_cast<int32_t>(members.size() - start);
      if (cnt >= min_freq)
        groups.push_back(VGroup{ref.size, start, cnt});
      else
        members.resize(start);
    }
    i = j;
  }

  // Step 3: size descending (stable: hash order among equal sizes).
  std::stable_sort(groups.begin(), groups.end(),
                   [](const VGroup &a, const VGroup &b) { return a.size > b.size; });

  // Step 4: greedy non-overlapping cover, for the coverage statistic.
  std::vector<uint8_t> marked(static_cast<size_t>(out.total_tokens), 0);
  const int64_t base = off[0];
  int64_t covered = 0, size_sum = 0;
  out.groups.reserve(groups.size());
  for (const VGroup &g : groups) {
    const Candidate &ref = members[g.first];
    out.groups.push_back(Detection::Group{ref.expr, ref.pos, g.size, g.count});
    size_sum += g.size;
    for (int32_t m = 0; m < g.count; ++m) {
      const Candidate &c = members[g.first + static_cast<size_t>(m)];
      uint8_t *h = marked.data() + (off[c.expr] - base) + c.pos;
      bool overlap = false;
      for (int q = 0; q < g.size && !overlap; ++q) overlap = h[q] != 0;
      if (overlap) continue;
      std::memset(h, 1, static_cast<size_t>(g.size));
      covered += g.size;
    }
  }
  out.covered_tokens = covered;
  out.avg_subtree_size =
      groups.empty() ? 0.0 : static_cast<double>(size_sum) / groups.size();
  out.coverage = out.total_tokens > 0
                     ? static_cast<double>(covered) / out.total_tokens
                     : 0.0;
}

int64_t mark_cached_subtrees(int E, const int32_t *tok, const double *val,
                             const int64_t *off, const SubtreeCache &cache,
                             int threads, int32_t *hints) {
  if (E <= 0) return 0;
  const int64_t base = off[0];
  std::vector<int64_t> removed(static_cast<size_t>(std::max(1, threads)), 0);
  const int nt = static_cast<int>(removed.size());
  parallel_for(nt, nt, [&](int64_t b, int64_t e) {
    std::vector<int32_t> sizes;
    for (int64_t c = b; c < e; ++c) {
      const int64_t x0 = E * c / nt, x1 = E * (c + 1) / nt;
      int64_t rem = 0;
      for (int64_t x = x0; x < x1; ++x) {
        const int len = static_cast<int>(off[x + 1] - off[x]);
        const int32_t *t = tok + off[x];
        const double *v = val + off[x];
        int32_t *h = hints + (off[x] - base);
        for (int i = 0; i < len; ++i) h[i] = -1;
        sizes.resize(static_cast<size_t>(len));
        subtree_sizes(t, len, sizes.data());
        for (int pos = 0; pos < len; ++pos) {
          if (h[pos] != -1) continue;
          const int size = sizes[pos];
          if (size < 3) continue;
          const auto it = cache.slot_of.find(flat_key(t + pos, v + pos, size));
          if (it == cache.slot_of.end()) continue;
          h[pos] = it->second;
          for (int k = 1; k < size; ++k) h[pos + k] = -2;
          rem += size - 1;
        }
      }
      removed[static_cast<size_t>(c)] = rem;
    }
  });
  int64_t total = 0;
  for (int64_t r : removed) total += r;
  return total;
}

}  // namespace sr
