// restart.cu -- restart files in the reference's layout (Restart.F90).
//
// The reference writes Fortran sequential unformatted files: every record
// is a 4-byte little-endian length, the payload, and the same length
// again.  Both of its layouts hold the same three kinds of record:
//   1. nstep (int32), time, delt, g, rho_0, scal1_0, Re, Pr, Sc (float64)
//      -- 68 bytes, packed (write_flow_big / write_flow_small, :470, :610);
//   2. the extents: SMALL (serial dump, write_flow_small) nxp2, nyp2, nzp2;
//      BIG (one file per rank, write_flow_big) sx, ex, sy, ey, sz, ez, the
//      interior index range of the rank (one rank here: 2..n+1);
//   3. u, v, w, p, rho, scal1, each the whole ghosted array
//      (nx+2)(ny+2)(nz+2) in Fortran order.
// Readers check the extents as Greadfile (:115-120) and start_big
// (:220-226) do.  A record of more than 2^31-1 bytes would need the
// compiler's subrecord convention and is refused.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "anel_internal.h"
#include "ns_solver.h"

namespace anel {

namespace {

constexpr int64_t kMaxRecord = 0x7fffffffLL;

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

bool put_record(FILE* f, const void* data, int64_t bytes) {
  const int32_t m = (int32_t)bytes;
  return std::fwrite(&m, 4, 1, f) == 1 && (bytes == 0 || std::fwrite(data, 1, (size_t)bytes, f) == (size_t)bytes) &&
         std::fwrite(&m, 4, 1, f) == 1;
}

// reads one record of exactly `bytes` bytes into data
int get_record(FILE* f, void* data, int64_t bytes, const char* what) {
  int32_t m0 = 0, m1 = 0;
  if (std::fread(&m0, 4, 1, f) != 1) {
    set_error("restart: end of file before the %s record", what);
    return ANEL_ERR_ARG;
  }
  if ((int64_t)m0 != bytes) {
    set_error("restart: the %s record holds %d bytes, expected %lld", what, m0, (long long)bytes);
    return ANEL_ERR_SIZE;
  }
  if (bytes && std::fread(data, 1, (size_t)bytes, f) != (size_t)bytes) {
    set_error("restart: the %s record is truncated", what);
    return ANEL_ERR_ARG;
  }
  if (std::fread(&m1, 4, 1, f) != 1 || m1 != m0) {
    set_error("restart: the %s record has no matching end marker", what);
    return ANEL_ERR_ARG;
  }
  return ANEL_OK;
}

void pack_header(const anel_restart_header& h, unsigned char* b) {
  std::memcpy(b, &h.nstep, 4);
  const double v[8] = {h.time, h.delt, h.g, h.rho_0, h.scal1_0, h.Re, h.Pr, h.Sc};
  std::memcpy(b + 4, v, 64);
}

void unpack_header(const unsigned char* b, anel_restart_header& h) {
  std::memcpy(&h.nstep, b, 4);
  double v[8];
  std::memcpy(v, b + 4, 64);
  h.time = v[0];
  h.delt = v[1];
  h.g = v[2];
  h.rho_0 = v[3];
  h.scal1_0 = v[4];
  h.Re = v[5];
  h.Pr = v[6];
  h.Sc = v[7];
}

int extents(int32_t layout, int32_t nx, int32_t ny, int32_t nz, int32_t* e, int* ne) {
  if (layout == ANEL_RESTART_SMALL) {
    e[0] = nx + 2;
    e[1] = ny + 2;
    e[2] = nz + 2;
    *ne = 3;
  } else if (layout == ANEL_RESTART_BIG) {
    const int32_t v[6] = {2, nx + 1, 2, ny + 1, 2, nz + 1};
    std::memcpy(e, v, sizeof(v));
    *ne = 6;
  } else {
    set_error("restart: layout must be ANEL_RESTART_SMALL or ANEL_RESTART_BIG");
    return ANEL_ERR_ARG;
  }
  return ANEL_OK;
}

int check_sizes(int32_t nx, int32_t ny, int32_t nz, int64_t* G) {
  if (nx < 1 || ny < 1 || nz < 1) {
    set_error("restart: sizes must be positive");
    return ANEL_ERR_SIZE;
  }
  *G = (int64_t)(nx + 2) * (ny + 2) * (nz + 2);
  if (*G * 8 > kMaxRecord) {
    set_error("restart: a field of %lld bytes exceeds one 2^31-1 byte record", (long long)(*G * 8));
    return ANEL_ERR_SIZE;
  }
  return ANEL_OK;
}

const char* const kNames[6] = {"u", "v", "w", "p", "rho", "scal1"};

}  // namespace
}  // namespace anel

using namespace anel;

extern "C" {

int anel_restart_write(const char* path, int32_t layout, const anel_restart_header* hdr, int32_t nx,
                       int32_t ny, int32_t nz, const double* const* fields) {
  if (!path || !hdr || !fields) {
    set_error("restart: null path, header or fields");
    return ANEL_ERR_ARG;
  }
  int64_t G = 0;
  int st = check_sizes(nx, ny, nz, &G);
  if (st != ANEL_OK) return st;
  int32_t e[6];
  int ne = 0;
  st = extents(layout, nx, ny, nz, e, &ne);
  if (st != ANEL_OK) return st;
  for (int q = 0; q < 6; ++q)
    if (!fields[q]) {
      set_error("restart: null %s", kNames[q]);
      return ANEL_ERR_ARG;
    }
  File F;
  F.f = std::fopen(path, "wb");
  if (!F.f) {
    set_error("restart: cannot open %s for writing", path);
    return ANEL_ERR_ARG;
  }
  unsigned char hb[68];
  pack_header(*hdr, hb);
  bool ok = put_record(F.f, hb, 68) && put_record(F.f, e, 4 * ne);
  for (int q = 0; q < 6 && ok; ++q) ok = put_record(F.f, fields[q], G * 8);
  if (!ok || std::fflush(F.f) != 0) {
    set_error("restart: write to %s failed", path);
    return ANEL_ERR_ARG;
  }
  return ANEL_OK;
}

int anel_restart_read(const char* path, int32_t layout, anel_restart_header* hdr, int32_t nx, int32_t ny,
                      int32_t nz, double* const* fields) {
  if (!path || !fields) {
    set_error("restart: null path or fields");
    return ANEL_ERR_ARG;
  }
  int64_t G = 0;
  int st = check_sizes(nx, ny, nz, &G);
  if (st != ANEL_OK) return st;
  int32_t e[6], r[6];
  int ne = 0;
  st = extents(layout, nx, ny, nz, e, &ne);
  if (st != ANEL_OK) return st;
  File F;
  F.f = std::fopen(path, "rb");
  if (!F.f) {
    set_error("restart: cannot open %s", path);
    return ANEL_ERR_ARG;
  }
  unsigned char hb[68];
  if ((st = get_record(F.f, hb, 68, "header")) != ANEL_OK) return st;
  if ((st = get_record(F.f, r, 4 * ne, "extents")) != ANEL_OK) return st;
  for (int q = 0; q < ne; ++q)
    if (r[q] != e[q]) {
      set_error("restart: the file's extent %d is %d, this run's is %d", q + 1, r[q], e[q]);
      return ANEL_ERR_SIZE;
    }
  for (int q = 0; q < 6; ++q) {
    if (!fields[q]) {
      set_error("restart: null %s", kNames[q]);
      return ANEL_ERR_ARG;
    }
    if ((st = get_record(F.f, fields[q], G * 8, kNames[q])) != ANEL_OK) return st;
  }
  if (hdr) unpack_header(hb, *hdr);
  return ANEL_OK;
}

int anel_ns_ctx_write_restart(anel_ns_ctx* ctx, const char* path, int32_t layout,
                              const anel_restart_header* hdr) {
  if (!ctx || !path || !hdr) return ANEL_ERR_ARG;
  NSSolver* s = ctx_solver(ctx);
  const int64_t G = s->ghosted_cells();
  std::vector<double> buf;
  try {
    buf.resize((size_t)G * 6);
  } catch (...) {
    set_error("restart: host buffer of %lld bytes", (long long)(G * 48));
    return ANEL_ERR_NOMEM;
  }
  anel_fields f{};
  f.u = buf.data();
  f.v = f.u + G;
  f.w = f.v + G;
  f.p = f.w + G;
  f.rho = f.p + G;
  f.scal1 = f.rho + G;
  int st = s->get_fields(&f, ANEL_MEM_HOST, nullptr);
  if (st != ANEL_OK) return st;
  const double* fl[6] = {f.u, f.v, f.w, f.p, f.rho, f.scal1};
  int nx, ny, nz;
  s->sizes(&nx, &ny, &nz);
  return anel_restart_write(path, layout, hdr, nx, ny, nz, fl);
}

int anel_ns_ctx_read_restart(anel_ns_ctx* ctx, const char* path, int32_t layout, int32_t icparam,
                             anel_restart_header* hdr) {
  if (!ctx || !path) return ANEL_ERR_ARG;
  NSSolver* s = ctx_solver(ctx);
  const int64_t G = s->ghosted_cells();
  std::vector<double> buf;
  try {
    buf.resize((size_t)G * 6);
  } catch (...) {
    set_error("restart: host buffer of %lld bytes", (long long)(G * 48));
    return ANEL_ERR_NOMEM;
  }
  double* fl[6];
  for (int q = 0; q < 6; ++q) fl[q] = buf.data() + (size_t)q * G;
  int nx, ny, nz;
  s->sizes(&nx, &ny, &nz);
  anel_restart_header h{};
  int st = anel_restart_read(path, layout, &h, nx, ny, nz, fl);
  if (st != ANEL_OK) return st;
  anel_fields f{};
  f.u = fl[0];
  f.v = fl[1];
  f.w = fl[2];
  f.p = fl[3];
  f.rho = fl[4];
  f.scal1 = fl[5];
  if ((st = s->set_fields(&f, ANEL_MEM_HOST, nullptr)) != ANEL_OK) return st;
  // start_small / start_big end with ghost() of the six fields (:425-430)
  if ((st = s->ghost_state(nullptr)) != ANEL_OK) return st;
  if (icparam) s->set_clock(h.time, h.nstep);
  if (hdr) *hdr = h;
  return ANEL_OK;
}

}  // extern "C"
