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

}  // namespace

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
  int header[kHdLength] = {0};
  header[0] = kHdVersion;
  header[1] = little_endian() ? 1 : 0;
  header[2] = npw;
  for (int j = 0; j < n_pdep_eigen; ++j) {
    const std::string fn = d + "/" + names[j];
    FILE* g = std::fopen(fn.c_str(), "wb");
    if (!g) return fail(WB_ERR_ARG, "cannot open " + fn + ": " + std::strerror(errno));
    bool w = std::fwrite(header, sizeof(int), kHdLength, g) == (size_t)kHdLength;
    w = w && std::fwrite(pdep + 2 * (size_t)j * ld, 2 * sizeof(double), npw, g) == (size_t)npw;
    std::fclose(g);
    if (!w) return fail(WB_ERR_ARG, "cannot write " + fn);
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
  for (int j = 0; j < nglob; ++j) {                    // pdep_read_G_and_distribute, pdep_io.f90:158-293
    const std::string fn = d + "/" + pdep_fname(j + 1, iq);
    FILE* g = std::fopen(fn.c_str(), "rb");
    if (!g) return fail(WB_ERR_ARG, "cannot open " + fn);
    int header[kHdLength];
    bool r = std::fread(header, sizeof(int), kHdLength, g) == (size_t)kHdLength;
    if (r && header[0] != kHdVersion) { std::fclose(g); return fail(WB_ERR_ARG, "unknown header version in " + fn); }
    if (r && header[2] != npw) { std::fclose(g); return fail(WB_ERR_ARG, "dimension mismatch in " + fn); }
    if (r && header[1] != (little_endian() ? 1 : 0)) { std::fclose(g); return fail(WB_ERR_ARG, "endianness mismatch in " + fn); }
    r = r && std::fread(pdep + 2 * (size_t)j * ld, 2 * sizeof(double), npw, g) == (size_t)npw;
    std::fclose(g);
    if (!r) return fail(WB_ERR_ARG, "short read of " + fn);
  }
  return WB_OK;
}
