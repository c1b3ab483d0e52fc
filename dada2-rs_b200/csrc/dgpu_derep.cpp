// Dereplication of a FASTQ file (plain or gzip) into the uniques the
// denoiser takes (src/derep.rs:43-240): identical sequences are grouped, each
// unique keeps its read count and the per-position SUM of its reads' Phred
// scores (deferred division), and the uniques are ordered by count
// descending, ties by sequence bytes ascending (the R derepFastq order).
// `map` gives each read's unique in input order.
//
// Reads are grouped in parallel by hash shard: every shard owns the
// sequences whose hash falls in it, so shards never share a unique and the
// final sort makes the result independent of the sharding.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <string>
#include <string_view>
#include <thread>
#include <unordered_map>
#include <vector>

#include <zlib.h>

#include "dada2_b200.h"
#include "dgpu_common.h"

struct dgpu_derep {
  std::vector<char> seq;        // uniques' bases back to back
  std::vector<uint32_t> off, len;
  std::vector<uint64_t> count;
  std::vector<uint32_t> qsum;   // per-position Phred sums, back to back like seq
  std::vector<uint32_t> map;    // per read: its unique
};

namespace {

struct Rec {
  uint64_t seq_off;
  uint64_t qual_off;
  uint32_t len;
};

int fail(int code, const std::string& msg) {
  dgpu::set_last_error(msg.c_str());
  return code;
}

// The whole file, decompressed when it is gzip (gzread passes plain files
// through unchanged).
int read_all(const char* path, std::vector<char>& buf) {
  gzFile f = gzopen(path, "rb");
  if (!f) return fail(DGPU_E_INVALID, std::string("cannot open ") + path);
  gzbuffer(f, 1 << 20);
  buf.clear();
  std::vector<char> chunk(size_t(1) << 22);
  for (;;) {
    const int got = gzread(f, chunk.data(), unsigned(chunk.size()));
    if (got < 0) {
      int e = 0;
      const std::string msg = gzerror(f, &e);
      gzclose(f);
      return fail(DGPU_E_INVALID, std::string("read error in ") + path + ": " + msg);
    }
    if (got == 0) break;
    buf.insert(buf.end(), chunk.data(), chunk.data() + got);
  }
  gzclose(f);
  return 0;
}

// Four-line records: @name, sequence, +[name], qualities of the same length.
int parse(const std::vector<char>& b, std::vector<Rec>& recs) {
  size_t p = 0;
  const size_t n = b.size();
  uint64_t rec_no = 0;
  auto line = [&](size_t& s, size_t& e) {
    s = p;
    while (p < n && b[p] != '\n') ++p;
    e = p;
    if (e > s && b[e - 1] == '\r') --e;
    if (p < n) ++p;
  };
  while (p < n) {
    size_t s0, e0, s1, e1, s2, e2, s3, e3;
    line(s0, e0);
    if (e0 == s0 && p >= n) break;  // trailing newline
    if (e0 == s0 || b[s0] != '@')
      return fail(DGPU_E_INVALID, "record " + std::to_string(rec_no) + ": header does not start with '@'");
    if (p >= n) return fail(DGPU_E_INVALID, "record " + std::to_string(rec_no) + ": truncated");
    line(s1, e1);
    line(s2, e2);
    if (e2 == s2 || b[s2] != '+')
      return fail(DGPU_E_INVALID, "record " + std::to_string(rec_no) + ": separator line does not start with '+'");
    line(s3, e3);
    if (e3 - s3 != e1 - s1)
      return fail(DGPU_E_INVALID, "record " + std::to_string(rec_no) + ": quality length differs from sequence length");
    recs.push_back(Rec{s1, s3, uint32_t(e1 - s1)});
    ++rec_no;
  }
  return 0;
}

struct Shard {
  std::unordered_map<std::string_view, uint32_t> index;
  std::vector<std::string_view> seq;
  std::vector<uint64_t> count;
  std::vector<std::vector<int64_t>> sums;
};

}  // namespace

extern "C" {

int dgpu_derep_fastq(const char* path, int phred_offset, int nthreads, dgpu_derep** out) {
  if (!path || !out) return fail(DGPU_E_INVALID, "null argument");
  std::vector<char> buf;
  if (int rc = read_all(path, buf)) return rc;
  std::vector<Rec> recs;
  if (int rc = parse(buf, recs)) return rc;
  const size_t nr = recs.size();
  int nt = nthreads > 0 ? nthreads : int(std::max(1u, std::thread::hardware_concurrency()));
  nt = int(std::min<size_t>(size_t(nt), std::max<size_t>(1, nr / 4096 + 1)));
  const size_t nshard = size_t(nt);
  // shard of each read by the hash of its sequence
  std::vector<uint32_t> shard_of(nr);
  auto run = [&](auto&& fn) {
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(fn, t);
    fn(0);
    for (auto& x : th) x.join();
  };
  run([&](int t) {
    for (size_t r = size_t(t); r < nr; r += size_t(nt)) {
      const std::string_view sv(buf.data() + recs[r].seq_off, recs[r].len);
      shard_of[r] = uint32_t(std::hash<std::string_view>{}(sv) % nshard);
    }
  });
  std::vector<Shard> shards(nshard);
  std::vector<uint32_t> local(nr);
  run([&](int t) {
    Shard& S = shards[size_t(t)];
    for (size_t r = 0; r < nr; ++r) {
      if (shard_of[r] != uint32_t(t)) continue;
      const Rec& R = recs[r];
      const std::string_view sv(buf.data() + R.seq_off, R.len);
      auto it = S.index.find(sv);
      uint32_t u;
      if (it == S.index.end()) {
        u = uint32_t(S.seq.size());
        S.index.emplace(sv, u);
        S.seq.push_back(sv);
        S.count.push_back(0);
        S.sums.emplace_back(R.len, 0);
      } else {
        u = it->second;
      }
      local[r] = u;
      S.count[u] += 1;
      int64_t* sum = S.sums[u].data();
      const unsigned char* q = reinterpret_cast<const unsigned char*>(buf.data() + R.qual_off);
      for (uint32_t j = 0; j < R.len; ++j) sum[j] += int64_t(q[j]) - int64_t(phred_offset);
    }
  });
  // every unique, ordered by count descending, then sequence ascending
  struct Key {
    uint32_t shard, idx;
  };
  std::vector<Key> all;
  for (size_t s = 0; s < nshard; ++s)
    for (uint32_t u = 0; u < shards[s].seq.size(); ++u) all.push_back(Key{uint32_t(s), u});
  std::sort(all.begin(), all.end(), [&](const Key& a, const Key& b) {
    const uint64_t ca = shards[a.shard].count[a.idx], cb = shards[b.shard].count[b.idx];
    if (ca != cb) return ca > cb;
    return shards[a.shard].seq[a.idx] < shards[b.shard].seq[b.idx];
  });
  dgpu_derep* D = new dgpu_derep();
  const size_t nu = all.size();
  std::vector<std::vector<uint32_t>> rank(nshard);
  for (size_t s = 0; s < nshard; ++s) rank[s].resize(shards[s].seq.size());
  uint64_t total = 0;
  for (size_t k = 0; k < nu; ++k) {
    rank[all[k].shard][all[k].idx] = uint32_t(k);
    total += shards[all[k].shard].seq[all[k].idx].size();
  }
  D->seq.resize(total);
  D->qsum.resize(total);
  D->off.resize(nu);
  D->len.resize(nu);
  D->count.resize(nu);
  uint64_t w = 0;
  for (size_t k = 0; k < nu; ++k) {
    const Shard& S = shards[all[k].shard];
    const std::string_view sv = S.seq[all[k].idx];
    D->off[k] = uint32_t(w);
    D->len[k] = uint32_t(sv.size());
    D->count[k] = S.count[all[k].idx];
    std::memcpy(D->seq.data() + w, sv.data(), sv.size());
    const std::vector<int64_t>& sum = S.sums[all[k].idx];
    for (size_t j = 0; j < sv.size(); ++j) {
      // the reference sums in f64 and stores round(sum) as u32: a negative
      // sum (scores below the offset) becomes 0, one above u32 is an error
      if (sum[j] > int64_t(UINT32_MAX)) {
        delete D;
        return fail(DGPU_E_UNSUPPORTED, "per-position Phred quality sum overflows u32");
      }
      D->qsum[w + j] = sum[j] < 0 ? 0u : uint32_t(sum[j]);
    }
    w += sv.size();
  }
  if (total >= 0xffffffffull) {
    delete D;
    return fail(DGPU_E_UNSUPPORTED, "more than 4 GiB of unique sequence");
  }
  D->map.resize(nr);
  for (size_t r = 0; r < nr; ++r) D->map[r] = rank[shard_of[r]][local[r]];
  *out = D;
  return 0;
}

int dgpu_derep_sizes(const dgpu_derep* d, int64_t* sizes) {
  if (!d || !sizes) return fail(DGPU_E_INVALID, "null argument");
  sizes[0] = int64_t(d->count.size());
  sizes[1] = int64_t(d->map.size());
  sizes[2] = int64_t(d->seq.size());
  return 0;
}

int dgpu_derep_fill(const dgpu_derep* d, char* seqs, uint32_t* offs, uint32_t* lens, uint64_t* counts,
                    uint32_t* qual_sums, uint32_t* map) {
  if (!d) return fail(DGPU_E_INVALID, "null argument");
  if (seqs) std::memcpy(seqs, d->seq.data(), d->seq.size());
  if (offs) std::memcpy(offs, d->off.data(), d->off.size() * 4);
  if (lens) std::memcpy(lens, d->len.data(), d->len.size() * 4);
  if (counts) std::memcpy(counts, d->count.data(), d->count.size() * 8);
  if (qual_sums) std::memcpy(qual_sums, d->qsum.data(), d->qsum.size() * 4);
  if (map) std::memcpy(map, d->map.data(), d->map.size() * 4);
  return 0;
}

void dgpu_derep_free(dgpu_derep* d) { delete d; }

}  // extern "C"
