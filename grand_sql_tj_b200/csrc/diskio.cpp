// The reference's checkpoint files (code/tjsq/block.f90:2760-3097), read and
// written on the host so that the library can take the blocks, truncations,
// bases and wavefunctions a Fortran run left on disk, and leave its own in
// the same form.
//
// Binary files are Fortran sequential unformatted files as gfortran and ifort
// write them: every WRITE statement is one record, framed by its length in
// bytes as a 4-byte little-endian integer before and after the data; default
// INTEGERs are 4 bytes, REAL(8) 8 bytes, arrays in column-major order.  A
// record above 2^31 - 9 bytes is written as subrecords whose leading markers
// are negative except for the last one and whose trailing markers are
// negative except for the first one.  Basis files are the formatted text of
// basis_to_disk (A4,I6 / A11,I4 / A13,I4 / A10,I4,2X,A12,I4 lines).
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/tj_b200.h"

int tjb_set_err(int code, const std::string &m);

namespace {

constexpr int64_t kMaxSub = 2147483639;   // the largest subrecord a Fortran runtime writes

struct File {
  FILE *f = nullptr;
  File(const char *path, const char *mode) { f = std::fopen(path, mode); }
  ~File() {
    if (f) std::fclose(f);
  }
};

// -------------------------------------------------------------- writing
bool put_marker(FILE *f, int32_t v) { return std::fwrite(&v, 4, 1, f) == 1; }

bool put_record(FILE *f, const void *data, int64_t n) {
  const char *p = (const char *)data;
  if (n <= kMaxSub) return put_marker(f, (int32_t)n) && (n == 0 || std::fwrite(p, 1, n, f) == (size_t)n) &&
                           put_marker(f, (int32_t)n);
  bool first = true;
  while (n > 0) {
    const int64_t m = n > kMaxSub ? kMaxSub : n;
    const bool last = m == n;
    if (!put_marker(f, last ? (int32_t)m : -(int32_t)m) || std::fwrite(p, 1, m, f) != (size_t)m ||
        !put_marker(f, first ? (int32_t)m : -(int32_t)m))
      return false;
    p += m;
    n -= m;
    first = false;
  }
  return true;
}
bool put_ints(FILE *f, std::initializer_list<int32_t> v) {
  std::vector<int32_t> a(v);
  return put_record(f, a.data(), (int64_t)a.size() * 4);
}

bool put_block(FILE *f, const tj_block &b) {
  if (!put_ints(f, {b.len}) || !put_ints(f, {b.num}) || !put_ints(f, {b.dim}) || !put_ints(f, {b.up_dif}) ||
      !put_ints(f, {b.down_dif}))
    return false;
  for (int i = 0; i < b.num; ++i) {
    const tj_block_sub &s = b.sub[i];
    if (!put_record(f, nullptr, 0) || !put_ints(f, {s.num_up, s.num_down, s.down_dif}) ||
        !put_ints(f, {s.row_dim, s.sdim}) || !put_record(f, b.data + s.off, (int64_t)s.row_dim * s.sdim * 8))
      return false;
  }
  return true;
}

// -------------------------------------------------------------- reading
struct Reader {
  FILE *f;
  std::string err;
  // one whole record (its subrecords joined); false at end of file or on a malformed frame
  bool record(std::vector<char> &out) {
    out.clear();
    bool first = true;
    for (;;) {
      int32_t head;
      if (std::fread(&head, 4, 1, f) != 1) {
        if (!first) err = "file ends inside a record";
        return false;
      }
      const bool more = head < 0;
      const int64_t n = more ? -(int64_t)head : head;
      const size_t at = out.size();
      out.resize(at + n);
      if (n > 0 && std::fread(out.data() + at, 1, n, f) != (size_t)n) {
        err = "file ends inside a record";
        return false;
      }
      int32_t tail;
      if (std::fread(&tail, 4, 1, f) != 1 || (tail < 0 ? -(int64_t)tail : tail) != n ||
          ((tail < 0) != !first)) {
        err = "record length markers disagree";
        return false;
      }
      first = false;
      if (!more) return true;
    }
  }
  bool ints(int32_t *v, int n) {
    std::vector<char> r;
    if (!record(r)) {
      if (err.empty()) err = "file ends early";
      return false;
    }
    if ((int64_t)r.size() != 4LL * n) {
      err = "record of " + std::to_string(r.size()) + " bytes where " + std::to_string(4 * n) + " were expected";
      return false;
    }
    std::memcpy(v, r.data(), r.size());
    return true;
  }
  bool skip_empty() {
    std::vector<char> r;
    if (!record(r)) {
      if (err.empty()) err = "file ends early";
      return false;
    }
    if (!r.empty()) {
      err = "non-empty record where an empty one was expected";
      return false;
    }
    return true;
  }
  bool doubles(double *dst, int64_t n) {
    std::vector<char> r;
    if (!record(r)) {
      if (err.empty()) err = "file ends early";
      return false;
    }
    if ((int64_t)r.size() != 8 * n) {
      err = "matrix record of " + std::to_string(r.size()) + " bytes where " + std::to_string(8 * n) + " were expected";
      return false;
    }
    if (dst && n) std::memcpy(dst, r.data(), r.size());
    return true;
  }
  bool at_end() {
    const int c = std::fgetc(f);
    if (c == EOF) return true;
    std::ungetc(c, f);
    return false;
  }
};

struct BlockHdr {
  int32_t len, num, dim, up_dif, down_dif;
  std::vector<tj_block_sub> subs;
  int64_t data_len = 0;
};
// block_from_disk (block.f90:2850-2870): header, then per sub-block an empty
// record, its labels, its dimensions and its matrix; data (when given) is
// written at data + data_off
bool get_block(Reader &r, BlockHdr &h, double *data, int64_t data_off) {
  if (!r.ints(&h.len, 1) || !r.ints(&h.num, 1) || !r.ints(&h.dim, 1) || !r.ints(&h.up_dif, 1) ||
      !r.ints(&h.down_dif, 1))
    return false;
  if (h.num < 0) {
    r.err = "negative sub-block count";
    return false;
  }
  h.subs.clear();
  h.data_len = 0;
  for (int i = 0; i < h.num; ++i) {
    int32_t lab[3], dims[2];
    if (!r.skip_empty() || !r.ints(lab, 3) || !r.ints(dims, 2)) return false;
    if (dims[0] < 0 || dims[1] < 0) {
      r.err = "negative sub-block dimension";
      return false;
    }
    const int64_t n = (int64_t)dims[0] * dims[1];
    tj_block_sub s;
    std::memset(&s, 0, sizeof s);
    s.num_up = lab[0];
    s.num_down = lab[1];
    s.down_dif = lab[2];
    s.row_dim = dims[0];
    s.sdim = dims[1];
    s.off = data_off + h.data_len;
    if (!r.doubles(data ? data + s.off : nullptr, n)) return false;
    h.subs.push_back(s);
    h.data_len += n;
  }
  return true;
}

int io_err(const char *what, const char *path, const std::string &why) {
  return tjb_set_err(TJ_ERR_ARG, std::string(what) + " " + (path ? path : "(null)") + ": " + why);
}

// ---------------------------------------------------------- basis text
bool read_line(FILE *f, std::string &s) {
  s.clear();
  int c;
  while ((c = std::fgetc(f)) != EOF && c != '\n') s.push_back((char)c);
  if (!s.empty() && s.back() == '\r') s.pop_back();
  return c != EOF || !s.empty();
}
// an integer field of `w` characters after a label of `a` characters
bool field(const std::string &s, int a, int w, int32_t &v) {
  if ((int)s.size() < a + 1) return false;
  std::string t = s.substr(a, w);
  char *end = nullptr;
  errno = 0;
  const long x = std::strtol(t.c_str(), &end, 10);
  if (end == t.c_str() || errno) return false;
  v = (int32_t)x;
  return true;
}

}  // namespace

extern "C" {

int tj_wave_to_disk(const char *path, const tj_wave *w) {
  if (!path || !w || (w->num > 0 && (!w->sub || !w->data))) return tjb_set_err(TJ_ERR_ARG, "tj_wave_to_disk: null argument");
  if (w->dim > INT32_MAX) return io_err("tj_wave_to_disk:", path, "dimension above a 4-byte integer");
  File F(path, "wb");
  if (!F.f) return io_err("tj_wave_to_disk: cannot open", path, std::strerror(errno));
  bool ok = put_ints(F.f, {w->sys_len}) && put_ints(F.f, {w->env_len}) && put_ints(F.f, {w->num}) &&
            put_ints(F.f, {(int32_t)w->dim});
  for (int i = 0; ok && i < w->num; ++i) {
    const tj_wave_sub &s = w->sub[i];
    ok = put_record(F.f, nullptr, 0) && put_ints(F.f, {s.sys_num_up, s.sys_num_down}) &&
         put_ints(F.f, {s.env_num_up, s.env_num_down}) && put_ints(F.f, {s.sys_dim, s.env_dim}) &&
         put_record(F.f, w->data + s.off, (int64_t)s.sys_dim * s.env_dim * 8);
  }
  if (!ok) return io_err("tj_wave_to_disk: write failed on", path, std::strerror(errno));
  return TJ_OK;
}

int tj_wave_from_disk(const char *path, tj_wave *hdr, tj_wave_sub *subs, double *data) {
  if (!path || !hdr) return tjb_set_err(TJ_ERR_ARG, "tj_wave_from_disk: null argument");
  File F(path, "rb");
  if (!F.f) return io_err("tj_wave_from_disk: cannot open", path, std::strerror(errno));
  Reader r{F.f, {}};
  int32_t sl, el, num, dim;
  if (!r.ints(&sl, 1) || !r.ints(&el, 1) || !r.ints(&num, 1) || !r.ints(&dim, 1))
    return io_err("tj_wave_from_disk:", path, r.err);
  if (num < 0 || dim < 0) return io_err("tj_wave_from_disk:", path, "negative sector count or dimension");
  const bool fill = subs && data;
  int64_t off = 0;
  for (int i = 0; i < num; ++i) {
    int32_t a[2], b[2], d[2];
    if (!r.skip_empty() || !r.ints(a, 2) || !r.ints(b, 2) || !r.ints(d, 2))
      return io_err("tj_wave_from_disk:", path, r.err);
    if (d[0] < 0 || d[1] < 0) return io_err("tj_wave_from_disk:", path, "negative sector dimension");
    const int64_t n = (int64_t)d[0] * d[1];
    if (off + n > dim) return io_err("tj_wave_from_disk:", path, "sectors exceed the stored dimension");
    if (fill) subs[i] = tj_wave_sub{a[0], a[1], b[0], b[1], d[0], d[1], off};
    if (!r.doubles(fill ? data + off : nullptr, n)) return io_err("tj_wave_from_disk:", path, r.err);
    off += n;
  }
  hdr->sys_len = sl;
  hdr->env_len = el;
  hdr->num = num;
  hdr->dim = dim;
  if (fill) {
    hdr->sub = subs;
    hdr->data = data;
  }
  return TJ_OK;
}

int tj_block_to_disk(const char *path, const tj_block *b) {
  if (!path || !b || (b->num > 0 && (!b->sub || !b->data))) return tjb_set_err(TJ_ERR_ARG, "tj_block_to_disk: null argument");
  File F(path, "wb");
  if (!F.f) return io_err("tj_block_to_disk: cannot open", path, std::strerror(errno));
  if (!put_block(F.f, *b)) return io_err("tj_block_to_disk: write failed on", path, std::strerror(errno));
  return TJ_OK;
}

int tj_block_from_disk(const char *path, tj_block_result *out) {
  if (!path || !out) return tjb_set_err(TJ_ERR_ARG, "tj_block_from_disk: null argument");
  File F(path, "rb");
  if (!F.f) return io_err("tj_block_from_disk: cannot open", path, std::strerror(errno));
  Reader r{F.f, {}};
  const bool fill = out->subs && out->data;
  BlockHdr h;
  if (!get_block(r, h, fill ? out->data : nullptr, 0)) return io_err("tj_block_from_disk:", path, r.err);
  out->num = h.num;
  out->data_len = h.data_len;
  if (fill) {
    std::memcpy(out->subs, h.subs.data(), h.subs.size() * sizeof(tj_block_sub));
    out->block = tj_block{h.len, h.num, h.dim, h.up_dif, h.down_dif, 0, out->subs, out->data};
  }
  return TJ_OK;
}

int tj_model_to_disk(const char *path, const tj_model *m) {
  if (!path || !m || m->nsub < 0 || (m->nsub > 0 && !m->sub)) return tjb_set_err(TJ_ERR_ARG, "tj_model_to_disk: null argument");
  File F(path, "wb");
  if (!F.f) return io_err("tj_model_to_disk: cannot open", path, std::strerror(errno));
  bool ok = put_ints(F.f, {m->len}) && put_block(F.f, m->ham);
  for (int i = 0; ok && i < m->nsub; ++i) {
    const tj_block_set &s = m->sub[i];
    ok = put_block(F.f, s.elec_up) && put_block(F.f, s.elec_down) && put_block(F.f, s.spin_sd) &&
         put_block(F.f, s.num_sn);
  }
  if (!ok) return io_err("tj_model_to_disk: write failed on", path, std::strerror(errno));
  return TJ_OK;
}

int tj_model_from_disk(const char *path, tj_model_result *out) {
  if (!path || !out) return tjb_set_err(TJ_ERR_ARG, "tj_model_from_disk: null argument");
  File F(path, "rb");
  if (!F.f) return io_err("tj_model_from_disk: cannot open", path, std::strerror(errno));
  Reader r{F.f, {}};
  const bool fill = out->sets && out->subs && out->data;
  int32_t len;
  if (!r.ints(&len, 1)) return io_err("tj_model_from_disk:", path, r.err);
  std::vector<BlockHdr> blocks;
  int64_t off = 0;
  while (!r.at_end()) {
    blocks.emplace_back();
    if (!get_block(r, blocks.back(), fill ? out->data : nullptr, off)) return io_err("tj_model_from_disk:", path, r.err);
    off += blocks.back().data_len;
  }
  if (blocks.empty() || (blocks.size() - 1) % 4 != 0)
    return io_err("tj_model_from_disk:", path, "not a Hamiltonian followed by whole operator sets");
  const int nsub = (int)(blocks.size() - 1) / 4;
  int nrec = 0;
  for (const auto &b : blocks) nrec += b.num;
  out->len = len;
  out->nsub = nsub;
  out->n_subs = nrec;
  out->data_len = off;
  if (!fill) return TJ_OK;
  int at = 0;
  auto view = [&](const BlockHdr &h) {
    std::memcpy(out->subs + at, h.subs.data(), h.subs.size() * sizeof(tj_block_sub));
    tj_block t{h.len, h.num, h.dim, h.up_dif, h.down_dif, 0, out->subs + at, out->data};
    at += h.num;
    return t;
  };
  out->model.len = len;
  out->model.nsub = nsub;
  out->model.ham = view(blocks[0]);
  for (int i = 0; i < nsub; ++i) {
    tj_block eu = view(blocks[1 + 4 * i]), ed = view(blocks[2 + 4 * i]), sd = view(blocks[3 + 4 * i]);
    tj_block sz{len, 0, 0, 0, 0, 0, out->subs + at, out->data};   // spin_sz is not stored
    tj_block sn = view(blocks[4 + 4 * i]);
    out->sets[i] = tj_block_set{eu, ed, sd, sz, sn};
  }
  out->model.sub = out->sets;
  return TJ_OK;
}

int tj_basis_to_disk(const char *path, const tj_basis *b) {
  if (!path || !b || (b->num > 0 && (!b->sub || !b->maps))) return tjb_set_err(TJ_ERR_ARG, "tj_basis_to_disk: null argument");
  File F(path, "w");
  if (!F.f) return io_err("tj_basis_to_disk: cannot open", path, std::strerror(errno));
  FILE *f = F.f;
  std::fprintf(f, "len=%6d\nnum=%6d\ndim=%6d\n", b->len, b->num, b->dim);
  for (int i = 0; i < b->num; ++i) {
    const tj_basis_map &m = b->sub[i];
    std::fprintf(f, "\nidx=%6d\nnum=%6d\ndim=%6d\nnew_num_up=%4d\nnew_num_down=%4d\n", m.idx, m.num, m.dim,
                 m.new_num_up, m.new_num_down);
    for (int x = 0; x < m.num; ++x) {
      const tj_basis_sub &s = b->maps[m.first + x];
      std::fprintf(f, "pos=%6d\ndim=%6d\nbl_num_up=%4d  bl_num_down=%4d\nst_num_up=%4d  st_num_down=%4d\n", s.spos,
                   s.sdim, s.bl_num_up, s.bl_num_down, s.st_num_up, s.st_num_down);
    }
  }
  if (std::ferror(f)) return io_err("tj_basis_to_disk: write failed on", path, std::strerror(errno));
  return TJ_OK;
}

int tj_basis_from_disk(const char *path, tj_basis_result *out) {
  if (!path || !out) return tjb_set_err(TJ_ERR_ARG, "tj_basis_from_disk: null argument");
  File F(path, "r");
  if (!F.f) return io_err("tj_basis_from_disk: cannot open", path, std::strerror(errno));
  FILE *f = F.f;
  std::string s;
  int32_t len, num, dim;
  auto line_int = [&](int a, int w, int32_t &v) { return read_line(f, s) && field(s, a, w, v); };
  if (!line_int(4, 6, len) || !line_int(4, 6, num) || !line_int(4, 6, dim) || num < 0)
    return io_err("tj_basis_from_disk:", path, "malformed header");
  const bool fill = out->sub && out->maps;
  int32_t nmaps = 0;
  for (int i = 0; i < num; ++i) {
    tj_basis_map m;
    std::memset(&m, 0, sizeof m);
    if (!read_line(f, s) || !line_int(4, 6, m.idx) || !line_int(4, 6, m.num) || !line_int(4, 6, m.dim) ||
        !line_int(11, 4, m.new_num_up) || !line_int(13, 4, m.new_num_down) || m.num < 0)
      return io_err("tj_basis_from_disk:", path, "malformed sector " + std::to_string(i + 1));
    m.first = nmaps;
    for (int x = 0; x < m.num; ++x) {
      tj_basis_sub q;
      std::memset(&q, 0, sizeof q);
      if (!line_int(4, 6, q.spos) || !line_int(4, 6, q.sdim) || !read_line(f, s) || !field(s, 10, 4, q.bl_num_up) ||
          !field(s, 28, 4, q.bl_num_down) || !read_line(f, s) || !field(s, 10, 4, q.st_num_up) ||
          !field(s, 28, 4, q.st_num_down))
        return io_err("tj_basis_from_disk:", path, "malformed sub-sector of sector " + std::to_string(i + 1));
      if (fill) out->maps[nmaps] = q;
      ++nmaps;
    }
    if (fill) out->sub[i] = m;
  }
  out->len = len;
  out->num = num;
  out->dim = dim;
  out->nmaps = nmaps;
  if (fill) out->basis = tj_basis{len, num, dim, 0, out->sub, out->maps};
  return TJ_OK;
}

int tj_disk_name(int kind, int idx, char *buf, int buflen) {
  static const char *names[7] = {"sysblocks", "systruns", "sysbs", "envblocks", "envtruns", "envbs", "eigvec"};
  if (kind < 0 || kind > 6 || idx < 1 || !buf || buflen < 1) return tjb_set_err(TJ_ERR_ARG, "tj_disk_name: bad argument");
  const int n = std::snprintf(buf, buflen, "%s%d", names[kind], idx);
  if (n < 0 || n >= buflen) return tjb_set_err(TJ_ERR_ARG, "tj_disk_name: buffer too short");
  return TJ_OK;
}

}  // extern "C"
