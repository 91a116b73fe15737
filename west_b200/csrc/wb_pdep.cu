// PDEP database I/O in WEST's format (host code).
//
// pdep_db_write (IO_kernel/pdep_db.f90:56-200) stores every PDEP eigenvector
// of q-point iq as a stream file Q<iq:9 digits>E<j:9 digits>.dat
// (generate_pdep_fname, pdep_db.f90:23-47) written by pdep_merge_and_write_G
// (IO_kernel/pdep_io.f90:35-150): a header of 32 int32 (HD_LENGTH,
// IO_kernel/mod_west_io.f90) with header(1) = 210405 (HD_VERSION),
// header(2) = 1 on a little-endian host, header(3) = the number of
// coefficients, then the complex128 G-space coefficients.  summary.json holds
// the cell (dielectric_matrix.domain.a1..a3 in bohr, b1..b3 in bohr^-1) and
// one dielectric_matrix.pdep entry per q-point with iq, q (crystal), eigenval
// and the eigenvector file names.  This build writes Gamma (one q-point) and
// rewrites summary.json with that single entry.
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <cstdint>
#include <sys/stat.h>

#include "wb_ctx.h"

using namespace wb;

namespace {

constexpr int kHdLength = 32;
constexpr int kHdVersion = 210405;

std::string pdep_fname(int j, int iq) {  // j, iq 1-based
  char b[32];
  std::snprintf(b, sizeof b, "Q%09dE%09d.dat", iq, j);
  return b;
}

bool little_endian() {
  const unsigned one = 1;
  unsigned char c;
  std::memcpy(&c, &one, 1);
  return c == 1;
}

void put_vec(std::string& o, const double* v, int n) {
  o += "[";
  char b[40];
  for (int i = 0; i < n; ++i) {
    std::snprintf(b, sizeof b, "%s%.17g", i ? ", " : "", v[i]);
    o += b;
  }
  o += "]";
}

// The numbers of the first JSON array that follows "key" (no nesting).
bool json_number_array(const std::string& txt, const char* key, std::vector<double>& out) {
  const std::string k = std::string("\"") + key + "\"";
  size_t p = txt.find(k);
  if (p == std::string::npos) return false;
  p = txt.find('[', p);
  const size_t e = txt.find(']', p);
  if (p == std::string::npos || e == std::string::npos) return false;
  out.clear();
  const char* s = txt.c_str() + p + 1;
  const char* end = txt.c_str() + e;
  while (s < end) {
    while (s < end && (std::isspace((unsigned char)*s) || *s == ',')) ++s;
    if (s >= end) break;
    char* q = nullptr;
    const double v = std::strtod(s, &q);
    if (q == s) return false;
    out.push_back(v);
    s = q;
  }
  return true;
}

// One eigenvector file (pdep_merge_and_write_G, pdep_io.f90:35-156): 32 int32
// header (version 210405, little-endian flag, npw), then npw complex128.
int write_vec(const std::string& fn, const double* v, int npw) {
  int header[kHdLength] = {0};
  header[0] = kHdVersion;
  header[1] = little_endian() ? 1 : 0;
  header[2] = npw;
  FILE* g = std::fopen(fn.c_str(), "wb");
  if (!g) return fail(WB_ERR_ARG, "cannot open " + fn + ": " + std::strerror(errno));
  bool w = std::fwrite(header, sizeof(int), kHdLength, g) == (size_t)kHdLength;
  w = w && std::fwrite(v, 2 * sizeof(double), npw, g) == (size_t)npw;
  std::fclose(g);
  return w ? WB_OK : fail(WB_ERR_ARG, "cannot write " + fn);
}

// pdep_read_G_and_distribute (pdep_io.f90:158-293), one rank
int read_vec(const std::string& fn, double* v, int npw) {
  FILE* g = std::fopen(fn.c_str(), "rb");
  if (!g) return fail(WB_ERR_ARG, "cannot open " + fn);
  int header[kHdLength];
  bool r = std::fread(header, sizeof(int), kHdLength, g) == (size_t)kHdLength;
  if (r && header[0] != kHdVersion) { std::fclose(g); return fail(WB_ERR_ARG, "unknown header version in " + fn); }
  if (r && header[2] != npw) { std::fclose(g); return fail(WB_ERR_ARG, "dimension mismatch in " + fn); }
  if (r && header[1] != (little_endian() ? 1 : 0)) { std::fclose(g); return fail(WB_ERR_ARG, "endianness mismatch in " + fn); }
  r = r && std::fread(v, 2 * sizeof(double), npw, g) == (size_t)npw;
  std::fclose(g);
  return r ? WB_OK : fail(WB_ERR_ARG, "short read of " + fn);
}

bool read_text(const std::string& fn, std::string& txt) {
  FILE* f = std::fopen(fn.c_str(), "r");
  if (!f) return false;
  char buf[4096];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) txt.append(buf, n);
  std::fclose(f);
  return true;
}

// The integer after "key": (top level, no nesting).
bool json_int(const std::string& txt, const char* key, int& out) {
  const std::string k = std::string("\"") + key + "\"";
  size_t p = txt.find(k);
  if (p == std::string::npos) return false;
  p = txt.find(':', p);
  if (p == std::string::npos) return false;
  char* q = nullptr;
  const long v = std::strtol(txt.c_str() + p + 1, &q, 10);
  if (q == txt.c_str() + p + 1) return false;
  out = (int)v;
  return true;
}

// The true/false values of the first JSON array after "key".
bool json_bool_array(const std::string& txt, const char* key, std::vector<int>& out) {
  const std::string k = std::string("\"") + key + "\"";
  size_t p = txt.find(k);
  if (p == std::string::npos) return false;
  p = txt.find('[', p);
  const size_t e = txt.find(']', p);
  if (p == std::string::npos || e == std::string::npos) return false;
  out.clear();
  for (size_t i = p + 1; i < e;) {
    if (txt.compare(i, 4, "true") == 0) { out.push_back(1); i += 4; }
    else if (txt.compare(i, 5, "false") == 0) { out.push_back(0); i += 5; }
    else ++i;
  }
  return true;
}

std::string restart_label(int j) {  // j 1-based, WRITE(my_label,'(i6.6)')
  char b[16];
  std::snprintf(b, sizeof b, "%06d", j);
  return b;
}

// One Fortran unformatted sequential record (4-byte length markers).
bool put_record(FILE* f, const double* v, size_t n) {
  const int32_t len = (int32_t)(n * sizeof(double));
  return std::fwrite(&len, 4, 1, f) == 1 && std::fwrite(v, sizeof(double), n, f) == n &&
         std::fwrite(&len, 4, 1, f) == 1;
}
bool get_record(FILE* f, double* v, size_t n) {
  int32_t a = 0, b = 0;
  if (std::fread(&a, 4, 1, f) != 1 || a != (int32_t)(n * sizeof(double))) return false;
  if (std::fread(v, sizeof(double), n, f) != n) return false;
  return std::fread(&b, 4, 1, f) == 1 && b == a;
}

}  // namespace

namespace wb {

int dav_restart_write(const char* dir, const DavRestart& r, int nvec, int nvecx, int npw, const double* dvg,
                      const double* dng, long ld) {
  const std::string d(dir);
  mkdir(dir, 0755);  // my_mkdir: an existing directory is fine
  std::string o = "{\n  \"dav_iter\": " + std::to_string(r.dav_iter) + ",\n  \"notcnv\": " +
                  std::to_string(r.notcnv) + ",\n  \"nbase\": " + std::to_string(r.nbase) + ",\n  \"conv\": [";
  for (int i = 0; i < nvec; ++i) o += std::string(i ? ", " : "") + (r.conv[i] ? "true" : "false");
  o += "],\n  \"ev\": ";
  put_vec(o, r.ev.data(), nvec);
  o += ",\n  \"ew\": ";
  put_vec(o, r.ew.data(), nvecx);
  o += "\n}\n";
  const std::string sf = d + "/summary.json";
  FILE* f = std::fopen(sf.c_str(), "w");
  if (!f) return fail(WB_ERR_ARG, "cannot open " + sf + ": " + std::strerror(errno));
  bool ok = std::fwrite(o.data(), 1, o.size(), f) == o.size();
  std::fclose(f);
  if (!ok) return fail(WB_ERR_ARG, "cannot write " + sf);
  const std::string hf = d + "/hr_vr.dat";  // one image: hr_distr then vr_distr
  FILE* h = std::fopen(hf.c_str(), "wb");
  if (!h) return fail(WB_ERR_ARG, "cannot open " + hf + ": " + std::strerror(errno));
  ok = put_record(h, r.hr.data(), (size_t)nvecx * nvecx) && put_record(h, r.vr.data(), (size_t)nvecx * nvecx);
  std::fclose(h);
  if (!ok) return fail(WB_ERR_ARG, "cannot write " + hf);
  for (int j = 0; j < r.nbase; ++j) {
    int rc = write_vec(d + "/V" + restart_label(j + 1) + ".dat", dvg + 2 * (size_t)j * ld, npw);
    if (!rc) rc = write_vec(d + "/N" + restart_label(j + 1) + ".dat", dng + 2 * (size_t)j * ld, npw);
    if (rc) return rc;
  }
  return WB_OK;
}

int dav_restart_read(const char* dir, DavRestart& r, int nvec, int nvecx, int npw, double* dvg, double* dng,
                     long ld) {
  const std::string d(dir);
  std::string txt;
  if (!read_text(d + "/summary.json", txt)) return fail(WB_ERR_ARG, "cannot open " + d + "/summary.json");
  std::vector<double> ev, ew;
  if (!json_int(txt, "dav_iter", r.dav_iter) || !json_int(txt, "notcnv", r.notcnv) ||
      !json_int(txt, "nbase", r.nbase) || !json_bool_array(txt, "conv", r.conv) ||
      !json_number_array(txt, "ev", ev) || !json_number_array(txt, "ew", ew))
    return fail(WB_ERR_ARG, "restart summary.json lacks dav_iter, notcnv, nbase, conv, ev or ew");
  if ((int)r.conv.size() != nvec || (int)ev.size() != nvec || (int)ew.size() != nvecx)
    return fail(WB_ERR_ARG, "restart written for another n_pdep_eigen or n_pdep_basis");
  if (r.nbase < 1 || r.nbase > nvecx || r.notcnv < 0 || r.notcnv > nvec || r.dav_iter < -1)
    return fail(WB_ERR_ARG, "restart summary.json holds an inconsistent state");
  r.ev = ev;
  r.ew = ew;
  r.hr.assign((size_t)nvecx * nvecx, 0.0);
  r.vr.assign((size_t)nvecx * nvecx, 0.0);
  const std::string hf = d + "/hr_vr.dat";
  FILE* h = std::fopen(hf.c_str(), "rb");
  if (!h) return fail(WB_ERR_ARG, "cannot open " + hf);
  const bool ok =
      get_record(h, r.hr.data(), (size_t)nvecx * nvecx) && get_record(h, r.vr.data(), (size_t)nvecx * nvecx);
  std::fclose(h);
  if (!ok) return fail(WB_ERR_ARG, hf + " is not two records of n_pdep_basis^2 doubles");
  for (int j = 0; j < r.nbase; ++j) {
    int rc = read_vec(d + "/V" + restart_label(j + 1) + ".dat", dvg + 2 * (size_t)j * ld, npw);
    if (!rc) rc = read_vec(d + "/N" + restart_label(j + 1) + ".dat", dng + 2 * (size_t)j * ld, npw);
    if (rc) return rc;
  }
  return WB_OK;
}

void dav_restart_clear(const char* dir, int nvecx) {  // davidson_restart_clear
  const std::string d(dir);
  std::remove((d + "/summary.json").c_str());
  std::remove((d + "/hr_vr.dat").c_str());
  for (int j = 1; j <= nvecx; ++j) {
    std::remove((d + "/V" + restart_label(j) + ".dat").c_str());
    std::remove((d + "/N" + restart_label(j) + ".dat").c_str());
  }
}

}  // namespace wb

extern "C" int wb_pdep_db_write(const char* dir, int iq, const double* q_cryst, const double* cell,
                                int n_pdep_eigen, const double* ev, const double* pdep, int ld, int npw) {
  if (!dir || !ev || !pdep || !cell) return fail(WB_ERR_ARG, "null argument");
  if (n_pdep_eigen < 1 || npw < 1 || ld < npw) return fail(WB_ERR_ARG, "bad sizes");
  if (iq != 1) return fail(WB_ERR_UNSUPPORTED, "only iq = 1 (Gamma) is written by this build");
  const std::string d(dir);
  std::vector<std::string> names(n_pdep_eigen);
  for (int j = 0; j < n_pdep_eigen; ++j) names[j] = pdep_fname(j + 1, iq);
  const double q0[3] = {0.0, 0.0, 0.0};
  const double* q = q_cryst ? q_cryst : q0;
  std::string o = "{\n \"dielectric_matrix\": {\n  \"domain\": {\n";
  const char* lab[6] = {"a1", "a2", "a3", "b1", "b2", "b3"};
  for (int i = 0; i < 6; ++i) {
    o += std::string("   \"") + lab[i] + "\": ";
    put_vec(o, cell + 3 * i, 3);
    o += i < 5 ? ",\n" : "\n";
  }
  o += "  },\n  \"pdep\": [\n   {\n    \"iq\": " + std::to_string(iq) + ",\n    \"q\": ";
  put_vec(o, q, 3);
  o += ",\n    \"eigenval\": ";
  put_vec(o, ev, n_pdep_eigen);
  o += ",\n    \"eigenvec\": [";
  for (int j = 0; j < n_pdep_eigen; ++j) o += (j ? ", \"" : "\"") + names[j] + "\"";
  o += "]\n   }\n  ]\n }\n}\n";
  const std::string sf = d + "/summary.json";
  FILE* f = std::fopen(sf.c_str(), "w");
  if (!f) return fail(WB_ERR_ARG, "cannot open " + sf + ": " + std::strerror(errno));
  const bool ok = std::fwrite(o.data(), 1, o.size(), f) == o.size();
  std::fclose(f);
  if (!ok) return fail(WB_ERR_ARG, "cannot write " + sf);
  for (int j = 0; j < n_pdep_eigen; ++j) {
    const int rc = write_vec(d + "/" + names[j], pdep + 2 * (size_t)j * ld, npw);
    if (rc) return rc;
  }
  return WB_OK;
}

extern "C" int wb_pdep_db_read(const char* dir, int iq, int nglob, double* ev, double* pdep, int ld, int npw) {
  if (!dir || !pdep) return fail(WB_ERR_ARG, "null argument");
  if (nglob < 1 || npw < 1 || ld < npw) return fail(WB_ERR_ARG, "bad sizes");
  if (iq != 1) return fail(WB_ERR_UNSUPPORTED, "only iq = 1 (Gamma) is read by this build");
  const std::string d(dir);
  if (ev) {
    const std::string sf = d + "/summary.json";
    FILE* f = std::fopen(sf.c_str(), "r");
    if (!f) return fail(WB_ERR_ARG, "cannot open " + sf);
    std::string txt;
    char buf[4096];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) txt.append(buf, n);
    std::fclose(f);
    std::vector<double> vals;
    if (!json_number_array(txt, "eigenval", vals) || (int)vals.size() < nglob)
      return fail(WB_ERR_ARG, "summary.json has fewer than the requested eigenvalues");
    for (int j = 0; j < nglob; ++j) ev[j] = vals[j];
  }
  for (int j = 0; j < nglob; ++j) {
    const int rc = read_vec(d + "/" + pdep_fname(j + 1, iq), pdep + 2 * (size_t)j * ld, npw);
    if (rc) return rc;
  }
  return WB_OK;
}
