// mles.cpp -- reader for the mesher's .mles files (include/cgx_mles.h).
//
// Restates, for one process, the record walk of StripedMesh::read_mles_
// (src/core/common/StripedMesh.hpp:1336-2380): a header at each offset, the
// record's data right after it, the next header `skip` bytes further on.  The
// data layouts per record follow the reference's readChunkedData calls:
//   no_fa_bf_cv_counts  idata pairs (nno, nbf, nfa, ncv, nno_p, nno_pb), then
//                       27 int8 face-zone counts            (:1605-1673)
//   *_I_AND_V_INT8      n int counts, then the int8 values  (:1782-1826, 1940-1985)
//   cvofa / cvobf       int8 pairs / int8                   (:1768-1780, 1925-1938)
//   *_D1, *_D2, DN33    n, 3n or 9n doubles, picked by name (:2021-2247)
//   zone headers        counts in idata pairs, geometry in rdata (:1712-1766, 2041-2055)

#include "../../include/cgx_mles.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <set>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

constexpr int32_t kMagic = 123581321;
enum : int32_t {
  ID_I0 = 11,
  ID_D0 = 12,
  ID_PARAMS = 91,
  ID_HASHIDS = 94,
  ID_EOF = 51,
  ID_FA_D2 = 25,
  ID_X_NO = 31,
  ID_PBI_PNO = 36,
  ID_CV_D1 = 42,
  ID_CV_D2 = 43,
  ID_CV_ZONE_HEADER = 46,
  ID_BF_ZONE_HEADER = 777,
  ID_SURFACE_PERIODIC_INFO = 802,
  ID_CVOBF_INT8 = 2004,
  ID_NOOBF_I_AND_V_INT8 = 2005,
  ID_CVOFA_INT8 = 2006,
  ID_NOOFA_I_AND_V_INT8 = 2007,
  ID_BF_D1 = 2120,
  ID_BF_D2 = 2121,
  ID_BF_DN33 = 2122,
  ID_PERIODIC_TRANSFORM = 4123,
  ID_NO_FA_BF_CV_COUNTS = 10001,
};
constexpr int32_t kFaZoneBoundary = 1, kCvZoneFluid = 1;

struct Header {
  char name[52];
  int32_t id;
  int64_t skip;
  int32_t idata[16];
  double rdata[12];
  uint64_t ui8data[4];
};
static_assert(sizeof(Header) == 256, "UGP header is 256 bytes");

// 64-bit count from an (lsw, msw) int pair, msw holding bits 31 and up
int64_t pair64(const int32_t* p) {
  int64_t lsw = p[0];
  const int64_t msw = p[1];
  if (lsw < 0) return lsw + 4294967296LL;  // writers that split at bit 32
  return (msw << 31) + lsw;
}

struct Error {
  int code;
  std::string what;
};

[[noreturn]] void fail(int code, const std::string& what) { throw Error{code, what}; }

struct File {
  FILE* f = nullptr;
  int64_t size = 0;  // bytes in the file
  ~File() {
    if (f) std::fclose(f);
  }
  // a record's data range [off, off + n*elem) must lie inside the file; checked
  // before anything of that size is allocated, so a small file cannot make the
  // reader allocate for counts it does not hold
  void need(int64_t off, int64_t n, int64_t elem, const char* what) const {
    if (off < 0 || n < 0 || n > (size - off) / elem)
      fail(CGX_MLES_E_IO, std::string(what) + " record runs past the end of the file (truncated?)");
  }
  void read_at(int64_t off, void* dst, size_t bytes) {
    if (bytes == 0) return;
    if (fseeko(f, off_t(off), SEEK_SET) != 0 || std::fread(dst, 1, bytes, f) != bytes)
      fail(CGX_MLES_E_IO, "short read at offset " + std::to_string(off));
  }
};

template <class T>
T* alloc(size_t n) {
  T* p = static_cast<T*>(std::malloc(sizeof(T) * (n ? n : 1)));
  if (!p) throw std::bad_alloc();
  return p;
}

// int8 indices in the file -> int, each checked against [0, limit)
int* read_indices(File& F, int64_t off, int64_t n, int64_t limit, const char* what) {
  F.need(off, n, int64_t(sizeof(int64_t)), what);
  std::vector<int64_t> tmp(static_cast<size_t>(n));
  F.read_at(off, tmp.data(), sizeof(int64_t) * size_t(n));
  int* out = alloc<int>(size_t(n));
  for (int64_t i = 0; i < n; ++i) {
    if (tmp[size_t(i)] < 0 || tmp[size_t(i)] >= limit) {
      std::free(out);
      fail(CGX_MLES_E_FORMAT, std::string(what) + " index out of range");
    }
    out[i] = int(tmp[size_t(i)]);
  }
  return out;
}

// counts (n ints) then values (int8): CSR offsets [n+1] and int values
void read_i_and_v(File& F, int64_t off, int64_t n, int64_t total, int64_t limit, int** csr, int** val,
                  const char* what) {
  F.need(off, n, int64_t(sizeof(int32_t)), what);
  std::vector<int32_t> cnt(static_cast<size_t>(n));
  F.read_at(off, cnt.data(), sizeof(int32_t) * size_t(n));
  int* c = alloc<int>(size_t(n) + 1);
  c[0] = 0;
  int64_t s = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (cnt[size_t(i)] < 0) {
      std::free(c);
      fail(CGX_MLES_E_FORMAT, std::string(what) + " negative count");
    }
    s += cnt[size_t(i)];
    if (s >= (int64_t(1) << 31)) {
      std::free(c);
      fail(CGX_MLES_E_UNSUPPORTED, std::string(what) + " too long for int offsets");
    }
    c[i + 1] = int(s);
  }
  if (s != total) {
    std::free(c);
    fail(CGX_MLES_E_FORMAT, std::string(what) + " total differs from its header");
  }
  *csr = c;
  *val = read_indices(F, off + int64_t(sizeof(int32_t)) * n, s, limit, what);
}

template <class T>
T* read_array(File& F, int64_t off, int64_t n) {
  F.need(off, n, int64_t(sizeof(T)), "array");
  T* p = alloc<T>(size_t(n));
  try {
    F.read_at(off, p, sizeof(T) * size_t(n));
  } catch (...) {
    std::free(p);
    throw;
  }
  return p;
}

bool is(const Header& h, const char* s) { return std::strncmp(h.name, s, sizeof(h.name)) == 0; }

void read_file(const char* path, cgx_mles* m) {
  File F;
  F.f = std::fopen(path, "rb");
  if (!F.f) fail(CGX_MLES_E_IO, std::string("cannot open ") + path);
  if (fseeko(F.f, 0, SEEK_END) != 0 || (F.size = int64_t(ftello(F.f))) < 0)
    fail(CGX_MLES_E_IO, std::string("cannot size ") + path);
  int32_t head[2];
  F.read_at(0, head, sizeof(head));
  if (head[0] != kMagic) {
    if (int32_t(__builtin_bswap32(uint32_t(head[0]))) == kMagic)
      fail(CGX_MLES_E_UNSUPPORTED, "byte-swapped file");
    fail(CGX_MLES_E_FORMAT, "not a UGP record file (magic number)");
  }
  if (head[1] != 5) fail(CGX_MLES_E_UNSUPPORTED, "io version " + std::to_string(head[1]) + " (5 is read)");
  m->io_version = head[1];

  bool have_counts = false;
  std::set<std::string> zone_names;
  std::vector<cgx_mles_bf_zone> zones;
  int64_t off = 8;
  for (int nrec = 0;; ++nrec) {
    if (nrec > 1000000) fail(CGX_MLES_E_FORMAT, "no end-of-file record");
    Header h;
    F.read_at(off, &h, sizeof(h));
    const int64_t data = off + int64_t(sizeof(Header));
    const bool needs_counts = h.id == ID_CVOBF_INT8 || h.id == ID_NOOBF_I_AND_V_INT8 || h.id == ID_CVOFA_INT8 ||
                              h.id == ID_NOOFA_I_AND_V_INT8 || h.id == ID_X_NO || h.id == ID_CV_D1 ||
                              h.id == ID_CV_D2 || h.id == ID_BF_D1 || h.id == ID_BF_D2 || h.id == ID_BF_DN33 ||
                              h.id == ID_FA_D2;
    if (needs_counts && !have_counts) fail(CGX_MLES_E_FORMAT, "data record before the counts record");
    switch (h.id) {
      case ID_NO_FA_BF_CV_COUNTS: {
        // one counts record only: the arrays already read are sized by it
        if (have_counts) fail(CGX_MLES_E_FORMAT, "a second counts record");
        m->nno = pair64(h.idata + 0);
        m->nbf = pair64(h.idata + 2);
        m->nfa = pair64(h.idata + 4);
        m->ncv = pair64(h.idata + 6);
        m->nno_p = pair64(h.idata + 8);
        m->nno_pb = pair64(h.idata + 10);
        F.read_at(data, m->nfa_zone, sizeof(m->nfa_zone));
        m->nfa_p = 0;
        for (int z = 0; z <= 25; ++z) m->nfa_p += m->nfa_zone[z];
        if (m->nfa_p + m->nfa_zone[26] != m->nfa) fail(CGX_MLES_E_FORMAT, "face-zone counts do not add up");
        const int64_t lim = (int64_t(1) << 31) - 1;
        if (m->nno < 0 || m->nbf < 0 || m->nfa < 0 || m->ncv <= 0 || m->nno > lim || m->nbf > lim ||
            m->nfa > lim || m->ncv > lim)
          fail(CGX_MLES_E_UNSUPPORTED, "counts outside int range");
        if (m->nno_p > 0 || m->nfa_p > 0) fail(CGX_MLES_E_UNSUPPORTED, "periodic mesh");
        have_counts = true;
        break;
      }
      case ID_PERIODIC_TRANSFORM:
      case ID_PBI_PNO:
      case ID_SURFACE_PERIODIC_INFO:
        fail(CGX_MLES_E_UNSUPPORTED, "periodic mesh");
      case ID_BF_ZONE_HEADER: {
        if (h.idata[0] != kFaZoneBoundary || h.idata[1] != int32_t(zones.size()))
          fail(CGX_MLES_E_FORMAT, "boundary zone header out of order");
        cgx_mles_bf_zone z;
        std::memset(&z, 0, sizeof(z));
        std::string name(h.name, strnlen(h.name, sizeof(h.name)));
        while (zone_names.count(name)) name += "1";  // unique names, as the reference makes them
        zone_names.insert(name);
        std::strncpy(z.name, name.c_str(), sizeof(z.name) - 1);
        z.nbf = pair64(h.idata + 2);
        z.ibf_f = pair64(h.idata + 6);
        z.area = h.rdata[0];
        z.area_over_delta = h.rdata[1];
        for (int k = 0; k < 3; ++k) {
          z.n[k] = h.rdata[2 + k];
          z.x[k] = h.rdata[5 + k];
        }
        zones.push_back(z);
        break;
      }
      case ID_CV_ZONE_HEADER:
        if (h.idata[0] != kCvZoneFluid) fail(CGX_MLES_E_FORMAT, "cell zone is not a fluid zone");
        if (m->ncv_zones < 16) m->cv_zone_ncv[m->ncv_zones] = pair64(h.idata + 2);
        ++m->ncv_zones;
        break;
      case ID_CVOBF_INT8:
        if (pair64(h.idata) != m->nbf || m->cvobf) fail(CGX_MLES_E_FORMAT, "cvobf record");
        m->cvobf = read_indices(F, data, m->nbf, m->ncv, "cvobf");
        break;
      case ID_NOOBF_I_AND_V_INT8:
        if (pair64(h.idata) != m->nbf || m->noobf_i) fail(CGX_MLES_E_FORMAT, "noobf record");
        read_i_and_v(F, data, m->nbf, pair64(h.idata + 2), m->nno, &m->noobf_i, &m->noobf_v, "noobf");
        break;
      case ID_CVOFA_INT8:
        if (pair64(h.idata) != m->nfa || h.idata[2] != 2 || m->cvofa) fail(CGX_MLES_E_FORMAT, "cvofa record");
        m->cvofa = reinterpret_cast<int(*)[2]>(read_indices(F, data, 2 * m->nfa, m->ncv, "cvofa"));
        break;
      case ID_NOOFA_I_AND_V_INT8:
        if (pair64(h.idata) != m->nfa || m->noofa_i) fail(CGX_MLES_E_FORMAT, "noofa record");
        read_i_and_v(F, data, m->nfa, pair64(h.idata + 2), m->nno, &m->noofa_i, &m->noofa_v, "noofa");
        break;
      case ID_X_NO:
        if (pair64(h.idata) != m->nno || h.idata[2] != 3 || m->x_no) fail(CGX_MLES_E_FORMAT, "x_no record");
        m->x_no = reinterpret_cast<double(*)[3]>(read_array<double>(F, data, 3 * m->nno));
        break;
      case ID_CV_D1:
        if (pair64(h.idata) != m->ncv) fail(CGX_MLES_E_FORMAT, "cell scalar record size");
        if (is(h, "vol_cv") || is(h, "VOL_VV") || is(h, "vol_vv")) {
          if (m->vol_cv) fail(CGX_MLES_E_FORMAT, "two volume records");
          m->vol_cv = read_array<double>(F, data, m->ncv);
        } else if (is(h, "r_vv")) {
          if (m->r_vv) fail(CGX_MLES_E_FORMAT, "two r_vv records");
          m->r_vv = read_array<double>(F, data, m->ncv);
        }
        break;
      case ID_CV_D2:
        if (pair64(h.idata) != m->ncv || h.idata[2] != 3) fail(CGX_MLES_E_FORMAT, "cell vector record size");
        if (is(h, "x_vv") || is(h, "X_VV")) {
          if (m->x_vv) fail(CGX_MLES_E_FORMAT, "two x_vv records");
          m->x_vv = reinterpret_cast<double(*)[3]>(read_array<double>(F, data, 3 * m->ncv));
        } else if (is(h, "x_cv")) {
          if (m->x_cv) fail(CGX_MLES_E_FORMAT, "two x_cv records");
          m->x_cv = reinterpret_cast<double(*)[3]>(read_array<double>(F, data, 3 * m->ncv));
        }
        break;
      case ID_BF_D1:
        if (pair64(h.idata) != m->nbf) fail(CGX_MLES_E_FORMAT, "boundary scalar record size");
        if (is(h, "area_bf")) {
          if (m->area_bf) fail(CGX_MLES_E_FORMAT, "two area_bf records");
          m->area_bf = read_array<double>(F, data, m->nbf);
        } else if (is(h, "area_over_delta_bf")) {
          if (m->area_over_delta_bf) fail(CGX_MLES_E_FORMAT, "two area_over_delta_bf records");
          m->area_over_delta_bf = read_array<double>(F, data, m->nbf);
        }
        break;
      case ID_BF_D2:
        if (pair64(h.idata) != m->nbf || h.idata[2] != 3) fail(CGX_MLES_E_FORMAT, "boundary vector record size");
        if (is(h, "n_bf")) {
          if (m->n_bf) fail(CGX_MLES_E_FORMAT, "two n_bf records");
          m->n_bf = reinterpret_cast<double(*)[3]>(read_array<double>(F, data, 3 * m->nbf));
        } else if (is(h, "x_bf")) {
          if (m->x_bf) fail(CGX_MLES_E_FORMAT, "two x_bf records");
          m->x_bf = reinterpret_cast<double(*)[3]>(read_array<double>(F, data, 3 * m->nbf));
        }
        break;
      case ID_BF_DN33:
        if (pair64(h.idata) != m->nbf || h.idata[2] != 3 || h.idata[3] != 3)
          fail(CGX_MLES_E_FORMAT, "boundary tensor record size");
        if (is(h, "Gij_bf")) {
          if (m->Gij_bf) fail(CGX_MLES_E_FORMAT, "two Gij_bf records");
          m->Gij_bf = reinterpret_cast<double(*)[3][3]>(read_array<double>(F, data, 9 * m->nbf));
        }
        break;
      case ID_FA_D2:
        if (pair64(h.idata) != m->nfa || h.idata[2] != 3) fail(CGX_MLES_E_FORMAT, "face vector record size");
        if (is(h, "n_fa")) {
          if (m->n_fa) fail(CGX_MLES_E_FORMAT, "two n_fa records");
          m->n_fa = reinterpret_cast<double(*)[3]>(read_array<double>(F, data, 3 * m->nfa));
        } else if (is(h, "x_fa")) {
          if (m->x_fa) fail(CGX_MLES_E_FORMAT, "two x_fa records");
          m->x_fa = reinterpret_cast<double(*)[3]>(read_array<double>(F, data, 3 * m->nfa));
        }
        break;
      default:
        break;  // timestamps, parameters, hash ids, surface, bounding boxes
    }
    if (h.id == ID_EOF) break;
    if (h.skip < int64_t(sizeof(Header))) fail(CGX_MLES_E_FORMAT, "record with a bad skip");
    off += h.skip;
  }
  if (!have_counts) fail(CGX_MLES_E_FORMAT, "no counts record");
  if (!m->cvofa || !m->n_fa || !m->x_fa || !m->vol_cv || !m->x_cv)
    fail(CGX_MLES_E_FORMAT, "missing cvofa, n_fa, x_fa, vol_cv or x_cv");
  if (m->nbf > 0 && (!m->cvobf || !m->n_bf)) fail(CGX_MLES_E_FORMAT, "missing cvobf or n_bf");
  int64_t zsum = 0;
  for (const auto& z : zones) {
    if (z.ibf_f != zsum || z.nbf < 0) fail(CGX_MLES_E_FORMAT, "boundary zones are not contiguous");
    zsum += z.nbf;
  }
  if (zsum != m->nbf) fail(CGX_MLES_E_FORMAT, "boundary zone sizes do not add up to nbf");
  m->nbf_zones = int(zones.size());
  m->bf_zones = alloc<cgx_mles_bf_zone>(zones.size());
  if (!zones.empty()) std::memcpy(m->bf_zones, zones.data(), sizeof(cgx_mles_bf_zone) * zones.size());
}

}  // namespace

extern "C" const char* cgx_mles_last_error(void) { return g_err.c_str(); }

namespace {

constexpr int32_t kSlesMagic = kMagic + 1;  // data file, not a restart (StaticSolver.cpp:7575)

// 64-bit count as the (lsw, msw) int pair pair64 reads
void set_pair64(int32_t* p, int64_t n) {
  p[0] = int32_t(n & 0x7fffffffLL);
  p[1] = int32_t(n >> 31);
}

struct Out {
  FILE* f = nullptr;
  ~Out() {
    if (f) std::fclose(f);
  }
  void put(const void* p, size_t bytes) {
    if (bytes && std::fwrite(p, 1, bytes, f) != bytes) fail(CGX_MLES_E_IO, "short write");
  }
  void header(const char* name, int32_t id, int64_t data_bytes, Header h) {
    std::memset(h.name, 0, sizeof(h.name));
    std::strncpy(h.name, name, sizeof(h.name) - 1);
    h.id = id;
    h.skip = int64_t(sizeof(Header)) + data_bytes;
    put(&h, sizeof(h));
  }
};

Header blank() {
  Header h;
  std::memset(&h, 0, sizeof(h));
  return h;
}

}  // namespace

extern "C" int cgx_sles_write(const char* path, long long ncv, int step, double time, const double* rho,
                              const double* u, const double* rhoE, const char* params) {
  if (!path || ncv < 0 || (ncv > 0 && (!rho || !u || !rhoE))) {
    g_err = "cgx_sles_write: null argument or negative size";
    return CGX_MLES_E_IO;
  }
  // written to a temporary name, then renamed over the target, as the
  // reference does (StaticSolver.cpp:7567-7569, 7632-7636)
  const std::string tmp = std::string(path) + ".tmp";
  try {
    {
      Out O;
      O.f = std::fopen(tmp.c_str(), "wb");
      if (!O.f) fail(CGX_MLES_E_IO, "cannot create " + tmp);
      const int32_t head[2] = {kSlesMagic, 5};
      O.put(head, sizeof(head));
      {
        Header h = blank();
        h.idata[0] = h.idata[1] = 20;
        O.header("UGP_IO_HASHIDS", ID_HASHIDS, 40, h);
        const unsigned char zeros[40] = {};
        O.put(zeros, sizeof(zeros));
      }
      {
        const std::string p = params ? params : "";
        Header h = blank();
        h.idata[0] = int32_t(p.size());
        O.header("UGP_IO_PARAMS", ID_PARAMS, int64_t(p.size()), h);
        O.put(p.data(), p.size());
      }
      auto cv_record = [&](const char* name, int32_t id, const double* v, int comps) {
        Header h = blank();
        set_pair64(h.idata, ncv);
        if (comps == 3) h.idata[2] = 3;
        O.header(name, id, int64_t(ncv) * comps * int64_t(sizeof(double)), h);
        O.put(v, size_t(ncv) * comps * sizeof(double));
      };
      cv_record("rho", ID_CV_D1, rho, 1);
      cv_record("rhoE", ID_CV_D1, rhoE, 1);
      {
        Header h = blank();
        h.idata[0] = step;
        O.header("step", ID_I0, 0, h);
      }
      {
        Header h = blank();
        h.rdata[0] = time;
        O.header("time", ID_D0, 0, h);
      }
      cv_record("u", ID_CV_D2, u, 3);
      O.header("EOF", ID_EOF, 0, blank());
      if (std::fflush(O.f) != 0) fail(CGX_MLES_E_IO, "cannot flush " + tmp);
    }
    if (std::rename(tmp.c_str(), path) != 0) fail(CGX_MLES_E_IO, std::string("cannot rename to ") + path);
  } catch (const Error& e) {
    std::remove(tmp.c_str());
    g_err = "cgx_sles_write: " + e.what;
    return e.code;
  }
  return CGX_MLES_OK;
}

extern "C" int cgx_sles_read(const char* path, long long ncv, int* step, double* time, double* rho, double* u,
                             double* rhoE) {
  if (!path || ncv < 0) {
    g_err = "cgx_sles_read: null argument or negative size";
    return CGX_MLES_E_IO;
  }
  try {
    File F;
    F.f = std::fopen(path, "rb");
    if (!F.f) fail(CGX_MLES_E_IO, std::string("cannot open ") + path);
    if (fseeko(F.f, 0, SEEK_END) != 0 || (F.size = int64_t(ftello(F.f))) < 0)
      fail(CGX_MLES_E_IO, std::string("cannot size ") + path);
    int32_t head[2];
    F.read_at(0, head, sizeof(head));
    if (head[0] != kSlesMagic) fail(CGX_MLES_E_FORMAT, "not a .sles data file (magic number)");
    if (head[1] != 5) fail(CGX_MLES_E_UNSUPPORTED, "io version " + std::to_string(head[1]) + " (5 is read)");
    bool got[5] = {false, false, false, false, false};  // rho, rhoE, u, step, time
    int64_t off = 8;
    for (int nrec = 0;; ++nrec) {
      if (nrec > 100000) fail(CGX_MLES_E_FORMAT, "no end-of-file record");
      Header h;
      F.read_at(off, &h, sizeof(h));
      const int64_t data = off + int64_t(sizeof(Header));
      if (h.id == ID_CV_D1 && (is(h, "rho") || is(h, "rhoE"))) {
        if (pair64(h.idata) != ncv) fail(CGX_MLES_E_FORMAT, "cell record size differs from the mesh");
        const bool e = is(h, "rhoE");
        F.need(data, ncv, 8, e ? "rhoE" : "rho");
        double* dst = e ? rhoE : rho;
        if (dst) F.read_at(data, dst, size_t(ncv) * sizeof(double));
        got[e ? 1 : 0] = true;
      } else if (h.id == ID_CV_D2 && is(h, "u")) {
        if (pair64(h.idata) != ncv || h.idata[2] != 3) fail(CGX_MLES_E_FORMAT, "u record size differs from the mesh");
        F.need(data, 3 * ncv, 8, "u");
        if (u) F.read_at(data, u, 3 * size_t(ncv) * sizeof(double));
        got[2] = true;
      } else if (h.id == ID_I0 && is(h, "step")) {
        if (step) *step = h.idata[0];
        got[3] = true;
      } else if (h.id == ID_D0 && is(h, "time")) {
        if (time) *time = h.rdata[0];
        got[4] = true;
      }
      if (h.id == ID_EOF) break;
      if (h.skip < int64_t(sizeof(Header))) fail(CGX_MLES_E_FORMAT, "record with a bad skip");
      off += h.skip;
    }
    if (!(got[0] && got[1] && got[2] && got[3] && got[4]))
      fail(CGX_MLES_E_FORMAT, "missing rho, rhoE, u, step or time");
  } catch (const Error& e) {
    g_err = "cgx_sles_read: " + e.what;
    return e.code;
  }
  return CGX_MLES_OK;
}

extern "C" void cgx_mles_free(cgx_mles* m) {
  if (!m) return;
  std::free(m->x_no);
  std::free(m->cvofa);
  std::free(m->noofa_i);
  std::free(m->noofa_v);
  std::free(m->n_fa);
  std::free(m->x_fa);
  std::free(m->cvobf);
  std::free(m->noobf_i);
  std::free(m->noobf_v);
  std::free(m->n_bf);
  std::free(m->x_bf);
  std::free(m->area_bf);
  std::free(m->area_over_delta_bf);
  std::free(m->Gij_bf);
  std::free(m->vol_cv);
  std::free(m->r_vv);
  std::free(m->x_vv);
  std::free(m->x_cv);
  std::free(m->bf_zones);
  std::free(m);
}

extern "C" int cgx_mles_read(const char* path, cgx_mles** out) {
  if (!path || !out) {
    g_err = "cgx_mles_read: null argument";
    return CGX_MLES_E_IO;
  }
  *out = nullptr;
  cgx_mles* m = static_cast<cgx_mles*>(std::calloc(1, sizeof(cgx_mles)));
  if (!m) {
    g_err = "cgx_mles_read: out of host memory";
    return CGX_MLES_E_OOM;
  }
  try {
    read_file(path, m);
  } catch (const Error& e) {
    g_err = "cgx_mles_read: " + e.what;
    cgx_mles_free(m);
    return e.code;
  } catch (const std::bad_alloc&) {
    g_err = "cgx_mles_read: out of host memory";
    cgx_mles_free(m);
    return CGX_MLES_E_OOM;
  }
  *out = m;
  return CGX_MLES_OK;
}
