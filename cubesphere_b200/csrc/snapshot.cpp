// Snapshots of a solve's state (checkpoint / resume).
//
// The reference keeps `time, dtcur, n_cc_components, filenum` in riemann.in
// (1000riemann_geomesh_cs_mhd.f:1798-1804, read back under RESTART at
// :1527-1666 with a consistency check) and the fields in Silo files through
// WRITEDATA / READDATA (not in its tree).  Here one self-describing binary
// file holds both:
//
//   bytes 0..7   magic "CSB2SNP1"
//   bytes 8..11  header length H (uint32, little endian)
//   H bytes      JSON header: format version, the mesh and physics
//                parameters the state belongs to, time, dtcur, step, the
//                arrays (name, components, doubles) and the FNV-1a 64-bit
//                hash of the payload
//   payload      U (8 components), entropy, Bxf, Byf, Bzf: FP64 little
//                endian, panel-box layout [comp][panel][box]
//
// Loading checks the magic, the parameters against the context and the
// hash, so a resumed solve continues bit for bit.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cs_internal.h"

namespace {

uint64_t fnv1a(const unsigned char* p, size_t n, uint64_t h) {
  for (size_t t = 0; t < n; ++t) {
    h ^= p[t];
    h *= 1099511628211ULL;
  }
  return h;
}
const uint64_t kFnvOffset = 1469598103934665603ULL;

std::string fmt_double(double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%.17g", v);
  return b;
}

bool find_num(const std::string& js, const char* key, double& out) {
  const std::string k = std::string("\"") + key + "\":";
  const size_t at = js.find(k);
  if (at == std::string::npos) return false;
  return std::sscanf(js.c_str() + at + k.size(), "%lf", &out) == 1;
}
bool find_str(const std::string& js, const char* key, std::string& out) {
  const std::string k = std::string("\"") + key + "\":\"";
  const size_t at = js.find(k);
  if (at == std::string::npos) return false;
  const size_t end = js.find('"', at + k.size());
  if (end == std::string::npos) return false;
  out = js.substr(at + k.size(), end - at - k.size());
  return true;
}

size_t box_points(const cs_params& p) { return (size_t)6 * cs::Box(p.ntp, p.nr, p.nghost).size(); }

}  // namespace

extern "C" {

int cs_snapshot_write_host(const char* path, const cs_params* p, const double* U, const double* ent,
                           const double* bxf, const double* byf, const double* bzf, double time, double dtcur,
                           int64_t step) {
  if (!path || !p || !U || !ent || !bxf || !byf || !bzf) return CS_ERR_ARG;
  const size_t n = box_points(*p);
  const double* arr[5] = {U, ent, bxf, byf, bzf};
  const size_t cnt[5] = {8 * n, n, n, n, n};
  uint64_t h = kFnvOffset;
  for (int a = 0; a < 5; ++a) h = fnv1a((const unsigned char*)arr[a], cnt[a] * sizeof(double), h);
  char hex[32];
  std::snprintf(hex, sizeof hex, "%016llx", (unsigned long long)h);
  std::string js = "{\"format\":\"cubesphere_b200 snapshot\",\"version\":1";
  js += ",\"ntp\":" + std::to_string(p->ntp) + ",\"nr\":" + std::to_string(p->nr) +
        ",\"nghost\":" + std::to_string(p->nghost) + ",\"radial_mesh\":" + std::to_string(p->radial_mesh);
  js += ",\"rmin\":" + fmt_double(p->rmin) + ",\"rmax\":" + fmt_double(p->rmax) +
        ",\"radial_ratio\":" + fmt_double(p->radial_ratio) + ",\"gamma\":" + fmt_double(p->gamma);
  js += ",\"rhofloor\":" + fmt_double(p->rhofloor) + ",\"prsfloor\":" + fmt_double(p->prsfloor) +
        ",\"smallnum\":" + fmt_double(p->smallnum) + ",\"cfl_coef\":" + fmt_double(p->cfl_coef) +
        ",\"flatten_coef\":" + fmt_double(p->flatten_coef) +
        ",\"prs_flatten_coef\":" + fmt_double(p->prs_flatten_coef) + ",\"gm\":" + fmt_double(p->gm) +
        ",\"bc_lower\":" + std::to_string(p->bc_lower) + ",\"bc_upper\":" + std::to_string(p->bc_upper);
  js += ",\"rk_scheme\":" + std::to_string(p->rk_scheme) + ",\"time\":" + fmt_double(time) +
        ",\"dtcur\":" + fmt_double(dtcur) + ",\"step\":" + std::to_string((long long)step);
  js += ",\"arrays\":[{\"name\":\"U\",\"components\":8,\"doubles\":" + std::to_string(cnt[0]) +
        "},{\"name\":\"entropy\",\"components\":1,\"doubles\":" + std::to_string(n) +
        "},{\"name\":\"Bxf\",\"components\":1,\"doubles\":" + std::to_string(n) +
        "},{\"name\":\"Byf\",\"components\":1,\"doubles\":" + std::to_string(n) +
        "},{\"name\":\"Bzf\",\"components\":1,\"doubles\":" + std::to_string(n) + "}]";
  js += ",\"layout\":\"[comp][panel][box], box index ((k+G)*NJ+(j+G))*NI+(i+G)\",\"endian\":\"little\"";
  js += ",\"fnv1a64\":\"" + std::string(hex) + "\"}";
  FILE* f = std::fopen(path, "wb");
  if (!f) return CS_ERR_ARG;
  const uint32_t hl = (uint32_t)js.size();
  bool ok = std::fwrite("CSB2SNP1", 1, 8, f) == 8 && std::fwrite(&hl, 4, 1, f) == 1 &&
            std::fwrite(js.data(), 1, js.size(), f) == js.size();
  for (int a = 0; ok && a < 5; ++a) ok = std::fwrite(arr[a], sizeof(double), cnt[a], f) == cnt[a];
  ok = (std::fclose(f) == 0) && ok;
  return ok ? CS_OK : CS_ERR_ARG;
}

int cs_snapshot_read_host(const char* path, const cs_params* p, double* U, double* ent, double* bxf, double* byf,
                          double* bzf, double* time, double* dtcur, int64_t* step) {
  if (!path || !p || !U || !ent || !bxf || !byf || !bzf || !time || !dtcur || !step) return CS_ERR_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return CS_ERR_ARG;
  char magic[8];
  uint32_t hl = 0;
  if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "CSB2SNP1", 8) != 0 || std::fread(&hl, 4, 1, f) != 1 ||
      hl > (1u << 20)) {
    std::fclose(f);
    return CS_ERR_ARG;
  }
  std::string js(hl, '\0');
  if (std::fread(&js[0], 1, hl, f) != hl) {
    std::fclose(f);
    return CS_ERR_ARG;
  }
  double v = 0;
  const struct {
    const char* key;
    double want;
  } checks[] = {{"ntp", (double)p->ntp},       {"nr", (double)p->nr},         {"nghost", (double)p->nghost},
                {"radial_mesh", (double)p->radial_mesh}, {"rmin", p->rmin}, {"rmax", p->rmax},
                {"radial_ratio", p->radial_ratio},       {"gamma", p->gamma},
                {"rhofloor", p->rhofloor},               {"prsfloor", p->prsfloor},
                {"smallnum", p->smallnum},               {"cfl_coef", p->cfl_coef},
                {"flatten_coef", p->flatten_coef},       {"prs_flatten_coef", p->prs_flatten_coef},
                {"gm", p->gm},                           {"bc_lower", (double)p->bc_lower},
                {"bc_upper", (double)p->bc_upper},       {"rk_scheme", (double)p->rk_scheme}};
  for (const auto& c : checks)
    if (!find_num(js, c.key, v) || v != c.want) {
      std::fclose(f);
      return CS_ERR_STATE;  // the snapshot belongs to another mesh or physics
    }
  double t = 0, d = 0, st = 0;
  std::string hex;
  if (!find_num(js, "time", t) || !find_num(js, "dtcur", d) || !find_num(js, "step", st) ||
      !find_str(js, "fnv1a64", hex)) {
    std::fclose(f);
    return CS_ERR_ARG;
  }
  const size_t n = box_points(*p);
  double* arr[5] = {U, ent, bxf, byf, bzf};
  const size_t cnt[5] = {8 * n, n, n, n, n};
  bool ok = true;
  for (int a = 0; ok && a < 5; ++a) ok = std::fread(arr[a], sizeof(double), cnt[a], f) == cnt[a];
  char extra;
  ok = ok && std::fread(&extra, 1, 1, f) == 0;
  std::fclose(f);
  if (!ok) return CS_ERR_ARG;
  uint64_t h = kFnvOffset;
  for (int a = 0; a < 5; ++a) h = fnv1a((const unsigned char*)arr[a], cnt[a] * sizeof(double), h);
  char got[32];
  std::snprintf(got, sizeof got, "%016llx", (unsigned long long)h);
  if (hex != got) return CS_ERR_NUMERIC;  // payload does not match its hash
  *time = t;
  *dtcur = d;
  *step = (int64_t)st;
  return CS_OK;
}

}  // extern "C"
