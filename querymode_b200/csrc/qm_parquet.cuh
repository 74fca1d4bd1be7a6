// Parquet column chunks -> a table: PLAIN-encoded numeric pages (data page
// v1 and v2) with optional definition levels, uncompressed.  Included at the
// end of qm_api.cu.  The page headers (Thrift compact protocol) and the run
// headers of the RLE / bit-packed hybrid definition levels are parsed on the
// host (a few bytes per page / run); presence bits, ranks and the values are
// expanded on the device.  Follows decodeParquetColumnChunk's PLAIN path
// (src/parquet-decode.ts:390-618), parsePageHeader (:239-276),
// decodeRleBitPacked (:119-188) and decodePlainValues (:280-386).

#include <condition_variable>
#include <functional>
#include <thread>

namespace {

// Thrift compact protocol reader with the reference's reading rules
// (ThriftReader, src/parquet.ts:44-183): varints of at most 5 bytes keep the
// low 32 bits; i32 fields are their zigzag as an int32; the buffer's end
// ends a struct; fields are told apart by id alone; unknown types take no
// bytes.  Positions may run past the end (the page then has no data).
struct ThriftIn {
  const uint8_t *b;
  int64_t n, pos;
  int32_t last = 0;
  std::vector<int32_t> stack;

  uint8_t byte_at(int64_t i) const { return i < n ? b[i] : 0; }  // JS reads undefined, 0 in bit operations
  uint32_t varint32() {
    uint32_t r = 0;
    int shift = 0;
    while (pos < n) {
      const uint8_t c = b[pos++];
      r |= (uint32_t)(c & 0x7f) << shift;
      if (!(c & 0x80)) return r;
      shift += 7;
      if (shift >= 35) return r;
    }
    return r;
  }
  int32_t zigzag32() {
    const uint32_t v = varint32();
    return (int32_t)((v >> 1) ^ (0u - (v & 1)));
  }
  void skip_varint64() {  // readVarint64: to the terminator or the end
    while (pos < n)
      if (!(b[pos++] & 0x80)) return;
  }
  // next field of the current struct: false at STOP or at the buffer's end
  bool field(int &id, int &type) {
    if (pos >= n) return false;
    const uint8_t h = b[pos++];
    if (h == 0) return false;
    type = h & 0x0f;
    const int delta = h >> 4;
    id = delta ? last + delta : zigzag32();
    last = id;
    return true;
  }
  void begin() {
    stack.push_back(last);
    last = 0;
  }
  void end() {
    last = stack.empty() ? 0 : stack.back();
    if (!stack.empty()) stack.pop_back();
  }
  // Types that consume a byte at least when the buffer has one left (bools in
  // the type nibble and unknown types take none).
  static bool takes_bytes(int type) { return type >= 3 && type <= 12; }
  // A list or map past the buffer's end changes nothing but the position,
  // which is past the end already: its remaining elements are not walked.
  void skip(int type, int depth = 0) {
    if (depth > 64) return;  // deeper nesting than any page header: treat as skipped
    switch (type) {
      case 3: pos += 1; break;
      case 4: case 5: varint32(); break;
      case 6: skip_varint64(); break;
      case 7: pos += 8; break;
      case 8: {
        const uint32_t len = varint32();
        pos += len;
        break;
      }
      case 9: case 10: {
        const uint8_t h = byte_at(pos++);
        uint32_t size = h >> 4;
        if (size == 15) size = varint32();
        if (!takes_bytes(h & 0x0f)) break;  // elements of no bytes: the loop would change nothing
        for (uint32_t i = 0; i < size && pos < n; i++) skip(h & 0x0f, depth + 1);
        break;
      }
      case 11: {
        const uint32_t size = varint32();
        if (size > 0) {
          const uint8_t kv = byte_at(pos++);
          if (!takes_bytes(kv >> 4) && !takes_bytes(kv & 0x0f)) break;
          for (uint32_t i = 0; i < size && pos < n; i++) {
            skip(kv >> 4, depth + 1);
            skip(kv & 0x0f, depth + 1);
          }
        }
        break;
      }
      case 12: {
        begin();
        int id, t;
        while (field(id, t)) skip(t, depth + 1);
        end();
        break;
      }
      default: break;  // bools (in the type nibble) and unknown types take no bytes
    }
  }
};

struct PqHeader {
  int type = 0;
  int64_t uncompressed = 0, compressed = 0, num_values = 0;
  int encoding = 0;
  int64_t def_len = 0, rep_len = 0;
  int64_t header_size = 0;
};

// parsePageHeader (src/parquet-decode.ts:239-276): fields 1-3, data page (5),
// dictionary page (7), v2 (8), each by field id whatever its type.
bool pq_page_header(const uint8_t *b, int64_t n, int64_t off, PqHeader &h) {
  ThriftIn r{b, n, off};
  int id, t;
  while (r.field(id, t)) {
    if (id == 1) h.type = r.zigzag32();
    else if (id == 2) h.uncompressed = r.zigzag32();
    else if (id == 3) h.compressed = r.zigzag32();
    else if (id == 5 || id == 7 || id == 8) {
      r.begin();
      int fid, ft;
      while (r.field(fid, ft)) {
        if (fid == 1) h.num_values = r.zigzag32();
        else if (id != 8 && fid == 2) h.encoding = r.zigzag32();
        else if (id == 8 && (fid == 2 || fid == 3)) r.zigzag32();
        else if (id == 8 && fid == 4) h.encoding = r.zigzag32();
        else if (id == 8 && fid == 5) h.def_len = r.zigzag32();
        else if (id == 8 && fid == 6) h.rep_len = r.zigzag32();
        else if (id == 8 && fid == 7) { /* is_compressed: in the type nibble */ }
        else r.skip(ft);
      }
      r.end();
    } else {
      r.skip(t);
    }
  }
  h.header_size = r.pos - off;
  return true;
}

// The varint of an RLE / bit-packed run header (readVarint, src/footer.ts:
// 183-200): to the terminator or the end, the low 32 bits.
uint32_t pq_run_varint(const uint8_t *b, int64_t end, int64_t &pos) {
  uint32_t r = 0;
  int shift = 0;
  while (pos < end) {
    const uint8_t c = b[pos++];
    if (shift < 32) r |= (uint32_t)(c & 0x7f) << shift;
    if (!(c & 0x80)) return r;
    shift += 7;
  }
  return r;
}

// Run headers of an RLE / bit-packed hybrid stream of bit width 1 holding at
// most max_values levels (decodeRleBitPacked, src/parquet-decode.ts:119-188):
// appended to runs with rows from row0.  A header's count is its value
// shifted as a signed 32-bit number, as the reference's `header >> 1`; a
// negative bit-packed count, after which the reference would step back and
// read the same bytes again without end, ends the stream.  Returns the
// levels the stream yields.
int64_t pq_def_runs(const uint8_t *b, int64_t start, int64_t end, int64_t max_values, int64_t row0,
                    std::vector<qm_pq_run> &runs, int64_t &present) {
  int64_t pos = start, got = 0;
  present = 0;
  while (pos < end && got < max_values) {
    const uint32_t header = pq_run_varint(b, end, pos);
    const int64_t half = (int64_t)((int32_t)header >> 1);
    qm_pq_run run{};
    run.row0 = row0 + got;
    if ((header & 1) == 0) {
      run.value = pos < end ? (b[pos] & 1) : 0;
      pos += 1;
      run.count = std::min(half, max_values - got);
      present += run.value && run.count > 0 ? run.count : 0;
    } else {
      if (half < 0) break;
      const int64_t groups = half;
      run.packed = 1;
      run.byte_off = pos;
      run.count = std::min(groups * 8, max_values - got);
      run.value = (int32_t)std::max<int64_t>(0, std::min<int64_t>(end - pos, groups));
      // levels past the bytes present read as 0: count over the bytes there are
      const int64_t nbytes = std::min<int64_t>(run.value, (run.count + 7) / 8);
      for (int64_t q = 0; q < nbytes; q++) {
        uint32_t byte = b[pos + q];
        if (q == (run.count - 1) / 8 && (run.count & 7)) byte &= (1u << (run.count & 7)) - 1;
        present += __builtin_popcount(byte);
      }
      pos += groups;
    }
    if (run.count > 0) {
      runs.push_back(run);
      got += run.count;
    }
  }
  return got;
}

// Run headers of the dictionary indices (bit width bw <= 32, at most
// max_values of them; decodeRleBitPacked as above): row0 of a run is its
// first index number; an RLE run keeps its value (ceil(bw / 8) little-endian
// bytes, masked), a bit-packed one its first byte.  Returns the indices
// yielded.
int64_t pq_index_runs(const uint8_t *b, int64_t start, int64_t end, int bw, int64_t max_values,
                      std::vector<qm_pq_run> &runs) {
  int64_t pos = start, got = 0;
  const uint64_t mask = bw >= 32 ? 0xffffffffull : ((1ull << bw) - 1);
  while (pos < end && got < max_values) {
    const uint32_t header = pq_run_varint(b, end, pos);
    const int64_t half = (int64_t)((int32_t)header >> 1);
    qm_pq_run run{};
    run.row0 = got;
    if ((header & 1) == 0) {
      uint64_t v = 0;
      for (int i = 0; i < (bw + 7) / 8 && pos < end; i++) v |= (uint64_t)b[pos++] << (8 * i);
      run.value = (int32_t)(uint32_t)(v & mask);
      run.count = std::min(half, max_values - got);
    } else {
      if (half < 0) break;
      run.packed = 1;
      run.byte_off = pos;
      run.count = std::min(half * 8, max_values - got);
      pos += (half * 8 * bw + 7) / 8;
    }
    if (run.count > 0) {
      runs.push_back(run);
      got += run.count;
    }
  }
  return got;
}

int pq_width(int dtype) { return dtype == QM_I64 || dtype == QM_F64 ? 8 : 4; }

// One column as the device decodes it: host byte segments laid end to end
// (each at a 16-byte aligned offset) in one device buffer, the page
// descriptors and level runs pointing into it.
struct PqSeg {
  const uint8_t *p;
  int64_t bytes, off;
};
struct PqColumn {
  std::vector<PqSeg> segs;
  int64_t bytes = 0;  // device buffer size
  std::vector<qm_pq_page> pages;
  std::vector<qm_pq_run> runs;
  std::vector<qm_pq_run> iruns;  // dictionary index runs
  int64_t rows = 0;
  // Device offset of a page's bytes.  A page that starts where the previous
  // one ended in host memory extends its segment (pages of one buffer, as a
  // reader fetched them, become one copy); a new segment starts at the next
  // offset with the host address's alignment modulo 16.
  int64_t add_seg(const uint8_t *p, int64_t n) {
    if (!segs.empty() && n > 0 && segs.back().p + segs.back().bytes == p) {
      PqSeg &g = segs.back();
      const int64_t off = g.off + g.bytes;
      g.bytes += n;
      bytes = off + n;
      return off;
    }
    const int64_t off = ((bytes + 15) & ~(int64_t)15) + (int64_t)((uintptr_t)p & 15);
    segs.push_back({p, n, off});
    bytes = off + n;
    return off;
  }
};

// Host parse of one Parquet column chunk (num_values values) into pages and
// definition-level runs appended to col, its bytes at device offset base.
// Dictionary pages set the dictionary of the data pages after them; data
// pages are PLAIN or dictionary indices (RLE_DICTIONARY, or RLE: encodings
// 8 and 3, as the reference reads them).
int pq_parse_chunk(qm_ctx *ctx, const char *name, int dtype, const uint8_t *b, int64_t n, int64_t num_values,
                   int64_t base, PqColumn &col) {
  const int w = pq_width(dtype);
  std::vector<qm_pq_run> &runs = col.runs;
  const size_t run_first = runs.size(), irun_first = col.iruns.size();
  int64_t pos = 0, rows = 0;
  const int64_t row_base = col.rows;
  bool have_dict = false;
  int64_t dict_off = 0, dict_n = 0;
  while (pos < n && rows < num_values) {
    PqHeader h;
    if (!pq_page_header(b, n, pos, h) || h.compressed <= 0) break;
    pos += h.header_size;
    // a page running past the chunk is cut at its end, and ends the chunk
    const int64_t data = pos, data_end = h.compressed < n - pos ? pos + h.compressed : n;
    pos = data_end;
    if (h.type != 0 && h.type != 2 && h.type != 3) continue;  // other page types are skipped
    if (h.compressed != h.uncompressed)
      return set_err(ctx, QM_ERR_UNSUPPORTED, "column %s: compressed pages (pass an uncompressed chunk)", name);
    if (h.type == 2) {  // DICTIONARY_PAGE: PLAIN values
      have_dict = true;
      dict_off = base + data;
      dict_n = std::min(std::max<int64_t>(h.num_values, 0), (data_end - data) / w);
      continue;
    }
    const bool is_dict = h.encoding == 8 || h.encoding == 3;
    if (!is_dict && h.encoding != 0)
      return set_err(ctx, QM_ERR_UNSUPPORTED, "column %s: page encoding %d (PLAIN or RLE_DICTIONARY)", name,
                     h.encoding);
    const int64_t len = data_end - data;
    qm_pq_page pg{};
    pg.row0 = row_base + rows;
    pg.run0 = pg.run1 = (int32_t)runs.size();
    int64_t plain = data;
    bool has_def = false;
    int64_t nonnull = 0;
    if (h.type == 0) {
      // v1: levels behind a 4-byte length, recognised as the reference does
      if (8 <= len) {
        int32_t plen;
        memcpy(&plen, b + data, 4);
        const int64_t max_def = std::max<int64_t>(64, (h.num_values + 3) / 4 + 8);
        if (plen > 0 && plen <= max_def && plen < len - 4) {
          bool level;
          if (is_dict && have_dict) {  // the byte after the levels must be the index bit width
            const int64_t after = data + 4 + plen;
            int expect = 0;
            while (((int64_t)1 << expect) < dict_n) expect++;
            level = after < data_end && b[after] == (dict_n <= 1 ? 0 : expect);
          } else {
            const int64_t rem = len - 4 - plen;
            level = rem >= 0 && rem <= h.num_values * w;
          }
          if (level) {
            pq_def_runs(b, data + 4, data + 4 + plen, h.num_values, pg.row0, runs, nonnull);
            plain = data + 4 + plen;
            has_def = true;
          }
        }
      }
    } else {
      // the level sections as the reference slices them (subarray: a
      // negative offset counts from the page's end, every offset is cut to it)
      auto jsx = [&](int64_t x) { return x < 0 ? std::max<int64_t>(len + x, 0) : std::min<int64_t>(x, len); };
      const int64_t lim = (int64_t)1 << 40;
      const int64_t rep = std::max(-lim, std::min(lim, h.rep_len)), def = std::max(-lim, std::min(lim, h.def_len));
      const int64_t d0 = jsx(rep), d1 = std::max(d0, jsx(rep + def));
      if (h.def_len > 0) {
        pq_def_runs(b, data + d0, data + d1, h.num_values, pg.row0, runs, nonnull);
        has_def = true;
      }
      plain = data + jsx(rep + def);
    }
    pg.run1 = (int32_t)runs.size();
    if (!has_def) {
      nonnull = h.num_values;
      pg.run1 = pg.run0;
    }
    if (is_dict) {
      if (!have_dict) {  // indices without a dictionary yield nothing
        runs.resize(pg.run0);
        continue;
      }
      pg.dict = 1;
      pg.dict_off = dict_off;
      pg.dict_n = dict_n;
      pg.data_end = base + data_end;
      pg.bw = plain < data_end ? b[plain] : 0;
      if (pg.bw > 32)
        return set_err(ctx, QM_ERR_UNSUPPORTED, "column %s: dictionary index bit width %d", name, pg.bw);
      pg.irun0 = pg.irun1 = (int32_t)col.iruns.size();
      if (pg.bw > 0) pg.n_idx = pq_index_runs(b, plain + 1, data_end, pg.bw, nonnull, col.iruns);
      pg.irun1 = (int32_t)col.iruns.size();
      pg.rows = h.num_values;
      pg.avail = pg.rows;
    } else {
      pg.val_off = base + plain;
      pg.avail = std::max<int64_t>(0, (data_end - plain) / w);
      if (has_def) {
        pg.rows = h.num_values;
        pg.avail = std::min(pg.avail, nonnull);  // decodePlainValues(plain, dtype, nonNullCount)
      } else {
        pg.rows = std::min(h.num_values, pg.avail);
      }
    }
    pg.rows = std::min(pg.rows, num_values - rows);
    if (pg.rows <= 0) {
      runs.resize(pg.run0);
      col.iruns.resize(pg.dict ? pg.irun0 : col.iruns.size());
      continue;
    }
    col.pages.push_back(pg);
    rows += pg.rows;
  }
  for (size_t i = run_first; i < runs.size(); i++) runs[i].byte_off += base;
  for (size_t i = irun_first; i < col.iruns.size(); i++) col.iruns[i].byte_off += base;
  col.rows += rows;
  return QM_OK;
}

// decodePage (src/decode.ts:251-331) for a numeric dtype: the rows a page
// yields, its validity bitmap as one bit-packed level run, where its values
// are.
void lance_page(const qm_page &pa, int w, int64_t base, PqColumn &col) {
  const int64_t rc = pa.row_count, nc = pa.null_count, n = pa.bytes;
  qm_pq_page pg{};
  pg.row0 = col.rows;
  pg.run0 = pg.run1 = (int32_t)col.runs.size();
  if (nc > 0 && rc > 0) {
    const int64_t bm = (rc + 7) / 8;
    if (n < bm) return;  // bitmap cut short: no rows
    if (pa.data_offset >= 0) {  // Lance v2: every row has a slot
      pg.slotted = 1;
      pg.val_off = base + pa.data_offset;
      pg.avail = std::max<int64_t>(0, n - pa.data_offset) / w;
      pg.rows = std::min(rc, pg.avail);
    } else {  // packed: rowCount - nullCount values after the bitmap
      pg.val_off = base + bm;
      pg.avail = std::max<int64_t>(0, std::min(rc - nc, (n - bm) / w));
      pg.rows = rc;
    }
    if (pg.rows <= 0) return;
    qm_pq_run run{};
    run.row0 = pg.row0;
    run.count = pg.rows;
    run.byte_off = base;
    run.packed = 1;
    run.value = (int32_t)std::min<int64_t>(bm, INT32_MAX);
    col.runs.push_back(run);
    pg.run1 = pg.run0 + 1;
  } else {
    pg.val_off = base;
    pg.avail = n / w;
    pg.rows = rc > 0 ? std::min(rc, pg.avail) : pg.avail;
    pg.avail = pg.rows;
    if (pg.rows <= 0) return;
  }
  col.pages.push_back(pg);
  col.rows += pg.rows;
}

// A few host threads that run one function together (fn(part) for every
// part), reused for every window of an upload.
class HostTeam {
 public:
  explicit HostTeam(int n) : n_(n) {
    for (int i = 1; i < n; i++) th_.emplace_back([this, i] { loop(i); });
  }
  ~HostTeam() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      quit_ = true;
    }
    cv_.notify_all();
    for (auto &t : th_) t.join();
  }
  int size() const { return n_; }
  void run(const std::function<void(int)> &fn) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &fn;
      pending_ = n_ - 1;
      gen_++;
    }
    cv_.notify_all();
    fn(0);
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [&] { return pending_ == 0; });
    fn_ = nullptr;
  }

 private:
  void loop(int i) {
    int64_t seen = 0;
    for (;;) {
      const std::function<void(int)> *fn;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return quit_ || gen_ != seen; });
        if (quit_) return;
        seen = gen_;
        fn = fn_;
      }
      (*fn)(i);
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (--pending_ == 0) done_.notify_one();
      }
    }
  }
  int n_;
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  const std::function<void(int)> *fn_ = nullptr;
  int pending_ = 0;
  int64_t gen_ = 0;
  bool quit_ = false;
};

// Bytes [a, e) of the column's image (segments at their offsets, zero
// between) into h.
void fill_window(const PqColumn &col, int64_t a, int64_t e, uint8_t *h, int64_t h0) {
  size_t j = std::upper_bound(col.segs.begin(), col.segs.end(), a,
                              [](int64_t x, const PqSeg &g) { return x < g.off; }) - col.segs.begin();
  if (j > 0) j--;
  int64_t filled = a;
  for (; j < col.segs.size() && col.segs[j].off < e; j++) {
    const PqSeg &g = col.segs[j];
    const int64_t s0 = std::max(a, g.off), s1 = std::min(e, g.off + g.bytes);
    if (s1 <= s0) continue;
    if (s0 > filled) memset(h + (filled - h0), 0, (size_t)(s0 - filled));
    memcpy(h + (s0 - h0), g.p + (s0 - g.off), (size_t)(s1 - s0));
    filled = s1;
  }
  if (e > filled) memset(h + (filled - h0), 0, (size_t)(e - filled));
}

// Host segments into the device buffer through two pinned staging buffers:
// the column's byte image goes over in windows, a team of host threads
// filling one buffer while the other is copied.
int upload_segments(qm_ctx *ctx, const PqColumn &col, uint8_t *dev, std::unique_ptr<HostTeam> &team_slot) {
  if (col.bytes <= 0) return QM_OK;
  // Segments in page-locked memory go over directly, without staging.
  bool pinned = true;
  for (const PqSeg &g : col.segs) {
    if (g.bytes <= 0) continue;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, g.p) != cudaSuccess || at.type != cudaMemoryTypeHost ||
        cudaPointerGetAttributes(&at, g.p + g.bytes - 1) != cudaSuccess || at.type != cudaMemoryTypeHost) {
      cudaGetLastError();
      pinned = false;
      break;
    }
  }
  if (pinned) {
    for (const PqSeg &g : col.segs)
      if (g.bytes > 0 && cudaMemcpyAsync(dev + g.off, g.p, (size_t)g.bytes, cudaMemcpyHostToDevice, ctx->stream) !=
                             cudaSuccess)
        return set_err(ctx, QM_ERR_CUDA, "page upload: %s", cudaGetErrorString(cudaGetLastError()));
    return QM_OK;  // the caller synchronises before its host vectors go
  }
  if (col.bytes >= ((int64_t)16 << 20) && !team_slot) {  // host threads fill the staging buffers
    const int hw = (int)std::thread::hardware_concurrency();
    team_slot.reset(new HostTeam(std::max(1, std::min(16, hw / 2))));
  }
  HostTeam *team = team_slot.get();
  const int64_t win = std::min<int64_t>(col.bytes, (int64_t)64 << 20);
  HostBuf hb[2];
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int rc = QM_OK;
  for (int k = 0; k < 2 && rc == QM_OK; k++) {
    if (!ctx->pool->acquire((size_t)win, hb[k])) rc = set_err(ctx, QM_ERR_OOM, "pinned staging (%lld bytes)", (long long)win);
    else if (cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming) != cudaSuccess) rc = QM_ERR_CUDA;
  }
  bool used[2] = {false, false};
  for (int64_t a = 0, k = 0; rc == QM_OK && a < col.bytes; a += win, k ^= 1) {
    const int64_t e = std::min(col.bytes, a + win);
    if (used[k] && cudaEventSynchronize(ev[k]) != cudaSuccess) rc = QM_ERR_CUDA;
    if (rc) break;
    uint8_t *h = (uint8_t *)hb[k].p;
    if (team && e - a >= ((int64_t)4 << 20)) {
      const int parts = team->size();
      team->run([&](int i) {
        const int64_t s0 = a + (e - a) * i / parts, s1 = a + (e - a) * (i + 1) / parts;
        if (s1 > s0) fill_window(col, s0, s1, h, a);
      });
    } else {
      fill_window(col, a, e, h, a);
    }
    if (cudaMemcpyAsync(dev + a, h, (size_t)(e - a), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
        cudaEventRecord(ev[k], ctx->stream) != cudaSuccess)
      rc = QM_ERR_CUDA;
    used[k] = true;
  }
  if (rc == QM_ERR_CUDA) set_err(ctx, QM_ERR_CUDA, "page upload: %s", cudaGetErrorString(cudaGetLastError()));
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess && rc == QM_OK)
    rc = set_err(ctx, QM_ERR_CUDA, "page upload: %s", cudaGetErrorString(cudaGetLastError()));
  for (int k = 0; k < 2; k++) {
    if (ev[k]) cudaEventDestroy(ev[k]);
    ctx->pool->release(hb[k]);
  }
  return rc;
}

int upload_host_bytes(qm_ctx *ctx, const void *src, size_t n, void *dst) {
  cudaPointerAttributes at;
  const bool pinned = cudaPointerGetAttributes(&at, src) == cudaSuccess && at.type == cudaMemoryTypeHost;
  cudaGetLastError();
  if (pinned || n < ((size_t)64 << 20)) {
    CK(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, ctx->stream));
    return QM_OK;
  }
  PqColumn col;
  col.segs.push_back({(const uint8_t *)src, (int64_t)n, 0});
  col.bytes = (int64_t)n;
  std::unique_ptr<HostTeam> team;
  return upload_segments(ctx, col, (uint8_t *)dst, team);
}

// Scratch of one call in blocks of the context's pool (no cudaMalloc /
// cudaFree per call once the pool holds them); back to the pool at the end,
// after the call's last synchronise.
struct PoolBuf {
  qm_ctx *ctx;
  void *p = nullptr;
  size_t block = 0, bytes = 0;
  explicit PoolBuf(qm_ctx *c) : ctx(c) {}
  PoolBuf(const PoolBuf &) = delete;
  PoolBuf &operator=(const PoolBuf &) = delete;
  ~PoolBuf() { drop(); }
  void drop() {
    if (p) col_release(ctx, p, block);
    p = nullptr;
    block = bytes = 0;
  }
  int ensure(size_t n) {
    if (p && bytes >= n) return QM_OK;
    drop();
    p = col_alloc(ctx, n, block);
    if (!p) return set_err(ctx, QM_ERR_OOM, "device scratch (%zu bytes)", n);
    bytes = block;
    return QM_OK;
  }
};

}  // namespace

extern "C" {

#define CKF(call)                                                                                   \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess) return fail(set_err(ctx, QM_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_))); \
  } while (0)

int qm_table_from_pages(qm_ctx *ctx, int32_t n_cols, const qm_page_column *cols, qm_table **out) {
  if (!ctx || !out || n_cols <= 0 || !cols) return set_err(ctx, QM_ERR_INVALID, "qm_table_from_pages: bad arguments");
  *out = nullptr;
  cudaSetDevice(ctx->device);
  qm_table *t = new qm_table();
  t->ctx = ctx;
  PoolBuf chunk(ctx), pgs(ctx), rns(ctx), present(ctx), counts(ctx), ranks(ctx), temp(ctx);
  std::unique_ptr<HostTeam> team;  // fills the staging buffers of large columns
  auto fail = [&](int rc) {
    qm_table_destroy(t);  // synchronises before the scratch goes back to the pool
    return rc;
  };
  for (int i = 0; i < n_cols; i++) {
    const qm_page_column &c = cols[i];
    if (!c.name || c.n_pages < 0 || (c.n_pages > 0 && !c.pages) ||
        (c.dtype != QM_I32 && c.dtype != QM_I64 && c.dtype != QM_F32 && c.dtype != QM_F64))
      return fail(set_err(ctx, QM_ERR_INVALID, "page column %d: bad descriptor", i));
    for (auto &e : t->cols)
      if (e.name == c.name) return fail(set_err(ctx, QM_ERR_INVALID, "duplicate column %s", c.name));
    const int w = pq_width(c.dtype);
    // the pages' value width and its widening into the column's cells
    int w_in = w, conv = 0;
    switch (c.page_type) {
      case QM_PT_SAME: break;
      case QM_PT_INT8: case QM_PT_UINT8: w_in = 1; conv = c.page_type; break;
      case QM_PT_INT16: case QM_PT_UINT16: case QM_PT_FLOAT16: w_in = 2; conv = c.page_type; break;
      case QM_PT_UINT32: w_in = 4; conv = c.page_type; break;
      default: return fail(set_err(ctx, QM_ERR_INVALID, "column %s: page type %d", c.name, c.page_type));
    }
    const int want = c.page_type == QM_PT_SAME     ? c.dtype
                     : c.page_type == QM_PT_UINT32  ? QM_F64
                     : c.page_type == QM_PT_FLOAT16 ? QM_F32
                                                    : QM_I32;
    if (want != c.dtype)
      return fail(set_err(ctx, QM_ERR_INVALID, "column %s: page type %d widens into dtype %d, not %d", c.name,
                          c.page_type, want, c.dtype));
    PqColumn pc;
    for (int k = 0; k < c.n_pages; k++) {
      const qm_page &pa = c.pages[k];
      if ((!pa.buf && pa.bytes > 0) || pa.bytes < 0 || pa.row_count < 0 || pa.null_count < 0 || pa.data_offset < -1)
        return fail(set_err(ctx, QM_ERR_INVALID, "column %s page %d: bad descriptor", c.name, k));
      if (pa.parquet && conv)
        return fail(set_err(ctx, QM_ERR_INVALID, "column %s: Parquet chunks hold the column's own dtype", c.name));
      const int64_t base = pc.add_seg(pa.buf, pa.bytes);
      if (pa.parquet) {
        int rc = pq_parse_chunk(ctx, c.name, c.dtype, pa.buf, pa.bytes, pa.row_count, base, pc);
        if (rc) return fail(rc);
      } else {
        lance_page(pa, w_in, base, pc);
      }
      if (pc.rows > 0xffffffffLL || pc.runs.size() > (size_t)INT32_MAX)
        return fail(set_err(ctx, QM_ERR_UNSUPPORTED, "tables are limited to 2^32-1 rows"));
    }
    const int64_t rows = pc.rows;
    if (i == 0) {
      t->n_rows = rows;
    } else if (rows != t->n_rows) {
      return fail(set_err(ctx, QM_ERR_INVALID, "column %s decodes to %lld rows, column %s to %lld", c.name,
                          (long long)rows, cols[0].name, (long long)t->n_rows));
    }
    const int64_t words = (rows + 31) / 32;
    size_t tb = 0;
    CKF(qm_launch_pq_decode(nullptr, nullptr, 0, nullptr, 0, nullptr, w, w_in, conv, rows, nullptr, nullptr, nullptr, nullptr, &tb,
                            nullptr, nullptr, ctx->sm_count, ctx->stream));
    int rc;
    if ((rc = chunk.ensure((size_t)pc.bytes + 16)) ||
        (rc = pgs.ensure(std::max<size_t>(pc.pages.size(), 1) * sizeof(qm_pq_page))) ||
        (rc = rns.ensure(std::max<size_t>(pc.runs.size() + pc.iruns.size(), 1) * sizeof(qm_pq_run))) ||
        (rc = present.ensure((size_t)(words + 1) * 4)) || (rc = counts.ensure((size_t)(words + 1) * 4)) ||
        (rc = ranks.ensure((size_t)(words + 1) * 8)) || (rc = temp.ensure(tb + 16)))
      return fail(rc);
    DevCol col;
    col.name = c.name;
    col.dtype = c.dtype;
    // NULLs come from definition levels, and from dictionary indices past
    // the dictionary
    bool has_dict = false;
    for (const auto &pg : pc.pages) has_dict = has_dict || pg.dict;
    const bool nullable = !pc.runs.empty() || has_dict;
    col.data = col_alloc(ctx, std::max<size_t>((size_t)rows * w, 16), col.data_block);
    col.own_data = col.data != nullptr;
    if (nullable) {
      col.nulls = (uint32_t *)col_alloc(ctx, (size_t)(words + 1) * 4, col.nulls_block);
      col.own_nulls = col.nulls != nullptr;
    }
    if (!col.data || (nullable && !col.nulls)) {
      free_col(ctx, col);
      return fail(set_err(ctx, QM_ERR_OOM, "column %s: device memory", c.name));
    }
    t->cols.push_back(col);
    if (nullable) CKF(cudaMemsetAsync(col.nulls, 0, (size_t)(words + 1) * 4, ctx->stream));  // + the padding word
    if ((rc = upload_segments(ctx, pc, (uint8_t *)chunk.p, team))) return fail(rc);
    if (!pc.pages.empty())
      CKF(cudaMemcpyAsync(pgs.p, pc.pages.data(), pc.pages.size() * sizeof(qm_pq_page), cudaMemcpyHostToDevice,
                         ctx->stream));
    if (!pc.runs.empty())
      CKF(cudaMemcpyAsync(rns.p, pc.runs.data(), pc.runs.size() * sizeof(qm_pq_run), cudaMemcpyHostToDevice,
                         ctx->stream));
    if (!pc.iruns.empty())  // the index runs after the level runs
      CKF(cudaMemcpyAsync((qm_pq_run *)rns.p + pc.runs.size(), pc.iruns.data(), pc.iruns.size() * sizeof(qm_pq_run),
                          cudaMemcpyHostToDevice, ctx->stream));
    size_t tbytes = temp.bytes;
    CKF(qm_launch_pq_decode((const uint8_t *)chunk.p, (const qm_pq_page *)pgs.p, (int)pc.pages.size(),
                           (const qm_pq_run *)rns.p, (int)pc.runs.size(),
                           has_dict ? (const qm_pq_run *)rns.p + pc.runs.size() : nullptr, w, w_in, conv, rows,
                           (uint32_t *)present.p, (uint32_t *)counts.p,
                           (uint64_t *)ranks.p, temp.p, &tbytes, (unsigned char *)col.data, col.nulls,
                           ctx->sm_count, ctx->stream));
    ctx->launches += pc.runs.empty() ? 1 : 5;
    CKF(cudaStreamSynchronize(ctx->stream));  // the host vectors above go out of scope
  }
  *out = t;
  return QM_OK;
}
#undef CKF

int qm_table_from_parquet(qm_ctx *ctx, int32_t n_cols, const qm_parquet_column *cols, qm_table **out) {
  if (!ctx || !out || n_cols <= 0 || !cols) return set_err(ctx, QM_ERR_INVALID, "qm_table_from_parquet: bad arguments");
  std::vector<qm_page> pages((size_t)n_cols);
  std::vector<qm_page_column> pc((size_t)n_cols);
  for (int i = 0; i < n_cols; i++) {
    const qm_parquet_column &c = cols[i];
    if (c.num_values < 0 || c.chunk_bytes < 0 || (!c.chunk && c.chunk_bytes > 0))
      return set_err(ctx, QM_ERR_INVALID, "parquet column %d: bad descriptor", i);
    pages[i] = qm_page{c.chunk, c.chunk_bytes, c.num_values, 0, -1, 1, 0};
    pc[i] = qm_page_column{c.name, c.dtype, 1, &pages[i]};
  }
  return qm_table_from_pages(ctx, n_cols, pc.data(), out);
}

int qm_table_read_column(const qm_table *t, int32_t col, void *values, uint8_t *null_bytes) {
  if (!t || col < 0 || col >= (int32_t)t->cols.size() || (!values && !null_bytes)) return QM_ERR_INVALID;
  qm_ctx *ctx = t->ctx;
  cudaSetDevice(ctx->device);
  const DevCol &c = t->cols[col];
  const int64_t n = t->n_rows;
  if (values && n)
    CK(cudaMemcpyAsync(values, c.data, (size_t)n * dtype_size(c.dtype), cudaMemcpyDeviceToHost, ctx->stream));
  std::vector<uint32_t> nb;
  if (null_bytes && c.nulls) {
    nb.resize((size_t)(n + 31) / 32);
    if (n) CK(cudaMemcpyAsync(nb.data(), c.nulls, nb.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  if (null_bytes)
    for (int64_t r = 0; r < n; r++) null_bytes[r] = c.nulls ? (uint8_t)((nb[r >> 5] >> (r & 31)) & 1) : 0;
  return QM_OK;
}

}  // extern "C"
