// The reference's file surface in host C++: the modset master file, the ESRI
// ASCII DEM, the forcing CSV, the initial state (initiation) and the
// Results/<t>.txt writer, around the device state of fx_capi.cu.
//
// Each reader keeps the reference's parsing rules, because they decide the
// numbers the solver sees:
//   * modset: JSON with // and /* */ comments (main.cpp:106-109), keys of
//     read_modset (read_functions.cpp:39-89); PRINT_STEP and H_MIN_TO_PRINT
//     are stored as unsigned long (GlobVar.h:102), ROUGNESS_HEIGHT as double;
//   * DEM: NROWS/NCOLS from the first two lines (common.cpp:131-149),
//     XLLCORNER/YLLCORNER as double, CELLSIZE and NODATA_VALUE as the first
//     integer token (read_functions.cpp:130-139); values as float
//     (read_functions.cpp:118,155), first data line into irow = NROWS;
//   * forcing: comma-separated, a token that is not a number reads 0, an
//     empty line ends the file, data row k (after the header) goes to table
//     row k, values stored as float (read_functions.cpp:256-272); the run
//     length is the last row's time truncated to an integer (main.cpp:181-192).
#include <algorithm>
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dirent.h>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <vector>

#include "../csrc/fx_internal.h"
#include "fluxos_gpu.h"

namespace {

// ---------------------------------------------------------------- JSON ----
struct JVal {
  enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
  bool b = false;
  double n = 0;
  std::string s;
  std::vector<JVal> a;
  std::map<std::string, JVal> o;
  const JVal* get(const char* k) const {
    if (kind != OBJ) return nullptr;
    auto it = o.find(k);
    return it == o.end() ? nullptr : &it->second;
  }
};

struct JParser {
  const std::string& t;
  size_t i = 0;
  std::string err;
  explicit JParser(const std::string& text) : t(text) {}
  void ws() {
    for (;;) {
      while (i < t.size() && isspace((unsigned char)t[i])) ++i;
      if (i + 1 < t.size() && t[i] == '/' && t[i + 1] == '/') {
        while (i < t.size() && t[i] != '\n') ++i;
      } else if (i + 1 < t.size() && t[i] == '/' && t[i + 1] == '*') {
        size_t e = t.find("*/", i + 2);
        i = (e == std::string::npos) ? t.size() : e + 2;
      } else {
        return;
      }
    }
  }
  bool fail(const char* m) {
    if (err.empty()) err = std::string(m) + " at offset " + std::to_string(i);
    return false;
  }
  bool str(std::string& out) {
    if (t[i] != '"') return fail("expected string");
    ++i;
    while (i < t.size() && t[i] != '"') {
      char ch = t[i++];
      if (ch == '\\' && i < t.size()) {
        char e = t[i++];
        switch (e) {
          case 'n': ch = '\n'; break;
          case 't': ch = '\t'; break;
          case 'r': ch = '\r'; break;
          case 'b': ch = '\b'; break;
          case 'f': ch = '\f'; break;
          case 'u': {
            unsigned v = (unsigned)strtoul(t.substr(i, 4).c_str(), nullptr, 16);
            i += 4;
            ch = v < 128 ? (char)v : '?';
            break;
          }
          default: ch = e;
        }
      }
      out.push_back(ch);
    }
    if (i >= t.size()) return fail("unterminated string");
    ++i;
    return true;
  }
  bool val(JVal& v) {
    ws();
    if (i >= t.size()) return fail("unexpected end");
    char ch = t[i];
    if (ch == '{') {
      v.kind = JVal::OBJ;
      ++i;
      ws();
      if (i < t.size() && t[i] == '}') {
        ++i;
        return true;
      }
      for (;;) {
        ws();
        std::string k;
        if (!str(k)) return false;
        ws();
        if (i >= t.size() || t[i] != ':') return fail("expected ':'");
        ++i;
        JVal x;
        if (!val(x)) return false;
        v.o[k] = std::move(x);
        ws();
        if (i < t.size() && t[i] == ',') {
          ++i;
          continue;
        }
        if (i < t.size() && t[i] == '}') {
          ++i;
          return true;
        }
        return fail("expected ',' or '}'");
      }
    }
    if (ch == '[') {
      v.kind = JVal::ARR;
      ++i;
      ws();
      if (i < t.size() && t[i] == ']') {
        ++i;
        return true;
      }
      for (;;) {
        JVal x;
        if (!val(x)) return false;
        v.a.push_back(std::move(x));
        ws();
        if (i < t.size() && t[i] == ',') {
          ++i;
          continue;
        }
        if (i < t.size() && t[i] == ']') {
          ++i;
          return true;
        }
        return fail("expected ',' or ']'");
      }
    }
    if (ch == '"') {
      v.kind = JVal::STR;
      return str(v.s);
    }
    if (!t.compare(i, 4, "true")) {
      v.kind = JVal::BOOL;
      v.b = true;
      i += 4;
      return true;
    }
    if (!t.compare(i, 5, "false")) {
      v.kind = JVal::BOOL;
      v.b = false;
      i += 5;
      return true;
    }
    if (!t.compare(i, 4, "null")) {
      v.kind = JVal::NUL;
      i += 4;
      return true;
    }
    char* end = nullptr;
    v.n = strtod(t.c_str() + i, &end);
    if (end == t.c_str() + i) return fail("bad value");
    v.kind = JVal::NUM;
    i = (size_t)(end - t.c_str());
    return true;
  }
};

// The first whitespace token that reads as an int / double
// (common.cpp:38-66: stringstream >> int accepts a leading integer prefix).
bool first_int(const std::string& line, long long* out) {
  std::stringstream ss(line);
  std::string tok;
  while (ss >> tok) {
    std::stringstream t(tok);
    long long v;
    if (t >> v) {
      *out = v;
      return true;
    }
  }
  return false;
}
bool first_double(const std::string& line, double* out) {
  std::stringstream ss(line);
  std::string tok;
  while (ss >> tok) {
    std::stringstream t(tok);
    double v;
    if (t >> v) {
      *out = v;
      return true;
    }
  }
  return false;
}

struct Modset {
  std::string dem_file, meteo_file, inflow_file, output_folder;
  bool restart = false, ade = false, has_meteo = false, has_inflow = false;
  unsigned long print_step = 0, h_min_print = 0;
  unsigned long inflow_x = 0, inflow_y = 0;  // DISCHARGE_LOCATION (GlobVar.h:100)
  double ks = 0.0, d_coef = 0.0;
  bool wintra = false;                           // EXTERNAL_MODULES.WINTRA.STATUS
  double soil_release_rate = 0.0, soil_conc_bckgrd = 0.0;  // GlobVar.h:95
};

// Numbers stored in unsigned long fields (GlobVar.h:102) truncate toward 0.
unsigned long as_ulong(const JVal* v) {
  if (!v) return 0;
  if (v->kind == JVal::NUM) return v->n < 0 ? 0ul : (unsigned long)v->n;
  if (v->kind == JVal::BOOL) return v->b ? 1ul : 0ul;
  return 0;
}
double as_double(const JVal* v) {
  if (!v) return 0.0;
  if (v->kind == JVal::NUM) return v->n;
  if (v->kind == JVal::BOOL) return v->b ? 1.0 : 0.0;
  return 0.0;
}
bool as_bool(const JVal* v) {
  if (!v) return false;
  if (v->kind == JVal::BOOL) return v->b;
  if (v->kind == JVal::NUM) return v->n != 0;
  return false;
}

int read_modset(const std::string& path, Modset& m, std::string& err) {
  std::ifstream f(path);
  if (!f) {
    err = "cannot open modset " + path;
    return FX_ERR_IO;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  std::string text = ss.str();
  JParser p(text);
  JVal root;
  if (!p.val(root) || root.kind != JVal::OBJ) {
    err = "modset " + path + " is not valid JSON: " + p.err;
    return FX_ERR_IO;
  }
  const JVal* v;
  if (!(v = root.get("DEM_FILE")) || v->kind != JVal::STR) {
    err = "modset: DEM_FILE missing";
    return FX_ERR_IO;
  }
  m.dem_file = v->s;
  m.restart = as_bool(root.get("RESTART"));
  const JVal* out = root.get("OUTPUT");
  if (!out || !out->get("OUTPUT_FOLDER") || out->get("OUTPUT_FOLDER")->kind != JVal::STR) {
    err = "modset: OUTPUT.OUTPUT_FOLDER missing";
    return FX_ERR_IO;
  }
  m.output_folder = out->get("OUTPUT_FOLDER")->s;
  m.print_step = as_ulong(out->get("PRINT_STEP"));
  m.h_min_print = as_ulong(out->get("H_MIN_TO_PRINT"));
  m.ks = as_double(root.get("ROUGNESS_HEIGHT"));
  const JVal* mods = root.get("EXTERNAL_MODULES");
  const JVal* ade = mods ? mods->get("ADE_TRANSPORT") : nullptr;
  m.ade = ade && as_bool(ade->get("STATUS"));
  if (m.ade) m.d_coef = as_double(ade->get("D_COEF"));
  // read_functions.cpp:46-47,65
  m.soil_release_rate = as_double(root.get("SOIL_RELEASE_RATE"));
  m.soil_conc_bckgrd = as_double(root.get("SOIL_CONC_BACKGROUND"));
  const JVal* wintra = mods ? mods->get("WINTRA") : nullptr;
  m.wintra = wintra && as_bool(wintra->get("STATUS"));
  if ((v = root.get("METEO_FILE")) && v->kind == JVal::STR) {
    m.meteo_file = v->s;
    m.has_meteo = !m.meteo_file.empty();
  }
  // INFLOW_FILE.FILENAME and DISCHARGE_LOCATION (read_functions.cpp:74-88)
  if (const JVal* inf = root.get("INFLOW_FILE")) {
    m.has_inflow = true;
    const JVal* fn = inf->get("FILENAME");
    const JVal* loc = inf->get("DISCHARGE_LOCATION");
    if (!fn || fn->kind != JVal::STR || !loc) {
      err = "modset: INFLOW_FILE needs FILENAME and DISCHARGE_LOCATION";
      return FX_ERR_IO;
    }
    m.inflow_file = fn->s;
    m.inflow_x = as_ulong(loc->get("X_COORDINATE"));
    m.inflow_y = as_ulong(loc->get("Y_COORDINATE"));
  }
  if (!m.has_meteo && !m.has_inflow) {
    err = "METEO_FILE or INFLOW_FILE must be provided in master file: " + path;
    return FX_ERR_IO;
  }
  return FX_OK;
}

struct Dem {
  int nrows = 0, ncols = 0, dxy = 0;
  double xll = 0, yll = 0, nodata = 0;
  std::vector<double> zb_raw;  // full grid, GlobVar layout, float-valued
};

int read_dem(const std::string& path, Dem& dm, std::string& err) {
  std::ifstream f(path);
  if (!f) {
    err = "cannot open DEM " + path;
    return FX_ERR_IO;
  }
  std::string line;
  long long nr = -1, nc = -1, v = 0;
  for (int k = 0; k < 2; ++k) {
    std::getline(f, line);
    std::string key = line.substr(0, 5);
    for (auto& ch : key) ch = (char)toupper((unsigned char)ch);
    if (first_int(line, &v)) {
      if (key == "NROWS") nr = v;
      else if (key == "NCOLS") nc = v;
    }
  }
  if (nr < 2 || nc < 2) {
    err = "DEM " + path + ": NROWS/NCOLS missing or < 2";
    return FX_ERR_IO;
  }
  dm.nrows = (int)nr;
  dm.ncols = (int)nc;
  std::getline(f, line);
  first_double(line, &dm.xll);
  std::getline(f, line);
  first_double(line, &dm.yll);
  std::getline(f, line);
  if (!first_int(line, &v) || v < 1) {
    err = "DEM " + path + ": CELLSIZE must be a positive integer";
    return FX_ERR_IO;
  }
  dm.dxy = (int)v;
  std::getline(f, line);
  if (!first_int(line, &v)) v = 0;
  dm.nodata = (double)(int)v;
  const size_t mr = (size_t)dm.nrows + 2, mc = (size_t)dm.ncols + 2;
  dm.zb_raw.assign(mr * mc, 0.0);
  long long irow = dm.nrows;
  while (std::getline(f, line)) {
    const char* p = line.c_str();
    long long icol = 1;
    for (;;) {
      while (*p == ' ' || *p == '\t' || *p == '\r') ++p;
      if (!*p) break;
      const char* te = p;
      while (*te && *te != ' ' && *te != '\t' && *te != '\r') ++te;
      std::string tok(p, te);
      char* end = nullptr;
      float val = strtof(tok.c_str(), &end);
      if (end != tok.c_str() && irow >= 0 && irow <= dm.nrows + 1 && icol <= dm.ncols + 1)
        dm.zb_raw[(size_t)icol * mr + (size_t)irow] = (double)val;
      ++icol;
      p = te;
    }
    --irow;
  }
  return FX_OK;
}

// Armadillo csv_ascii load as the reference uses it (see file comment).
std::vector<std::vector<double>> read_csv_numbers(const std::string& path, bool* ok) {
  std::vector<std::vector<double>> rows;
  std::ifstream f(path);
  *ok = (bool)f;
  if (!f) return rows;
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty()) break;
    std::vector<double> r;
    std::stringstream ss(line);
    std::string tok;
    while (std::getline(ss, tok, ',')) {
      const char* s = tok.c_str();
      char* end = nullptr;
      double val = strtod(s, &end);
      bool good = end != s;
      if (good)
        while (*end == ' ' || *end == '\t' || *end == '\r') ++end;
      r.push_back(good && *end == '\0' ? val : 0.0);
    }
    rows.push_back(r);
  }
  return rows;
}

// read_inflow (read_functions.cpp:284-326): data row a (1-based after the
// header) goes to table row a - 1, columns t [s], discharge [m^3/s],
// concentration, stored as float. `tlast` is the last data row's time, the
// value read_inflow returns for ntim.
int read_inflow_table(const Modset& m, std::vector<float>& tab, double* tlast, std::string& err) {
  tab.assign(3 * (size_t)FX_METEO_ROWS, 0.0f);
  *tlast = 0.0;
  bool ok = false;
  auto rows = read_csv_numbers(m.inflow_file, &ok);
  if (!ok) {
    err = "cannot open INFLOW_FILE " + m.inflow_file;
    return FX_ERR_IO;
  }
  if (rows.size() > (size_t)FX_METEO_ROWS + 1) {
    err = "INFLOW_FILE has more than " + std::to_string(FX_METEO_ROWS) + " rows";
    return FX_ERR_ARG;
  }
  for (size_t a = 1; a < rows.size(); ++a) {
    for (int col = 0; col < 3; ++col)
      tab[(size_t)col * FX_METEO_ROWS + a - 1] = (float)(col < (int)rows[a].size() ? rows[a][col] : 0.0);
    *tlast = rows[a].empty() ? 0.0 : rows[a][0];
  }
  return FX_OK;
}

// read_geo's discharge cell (read_functions.cpp:228-231): round(coordinate -
// corner) / dxy, truncated into an unsigned long. The reference leaves the
// cell unset when both coordinates are 0 and indexes outside the grid for a
// location off the DEM; both are refused here.
int inflow_cell(const Modset& m, double xll, double yll, int dxy, int nrows, int ncols, int* irow,
                int* icol, std::string& err) {
  const double r = std::round((double)m.inflow_y - yll) / (double)dxy;
  const double q = std::round((double)m.inflow_x - xll) / (double)dxy;
  if ((m.inflow_x == 0 && m.inflow_y == 0) || !(r >= 1.0) || !(q >= 1.0) || r >= nrows + 1.0 ||
      q >= ncols + 1.0) {
    err = "INFLOW_FILE: DISCHARGE_LOCATION (" + std::to_string(m.inflow_x) + ", " +
          std::to_string(m.inflow_y) + ") is not an interior cell of the DEM";
    return FX_ERR_ARG;
  }
  *irow = (int)(unsigned long)r;
  *icol = (int)(unsigned long)q;
  return FX_OK;
}

// read_geo's wall / ks step (read_functions.cpp:175-225) and initiation's
// bed averaging, zero initial state and ghost ring (initiate.cpp:43-107,
// 159-228). Outputs are full GlobVar grids.
struct InitState {
  std::vector<double> zb, z, h, qx, qy, ks, twet, conc0, soil;
  std::vector<float> ldry, wall;
};

void initiate_bed(int NR, int NC, double nodata, double ks_input, bool ade, const double* zb_raw,
                  InitState& s) {
  const size_t mr = (size_t)NR + 2, mc = (size_t)NC + 2, n = mr * mc;
  auto IX = [mr](long r, long c) { return (size_t)c * mr + (size_t)r; };
  s.zb.assign(n, 0.0);
  s.z.assign(n, 0.0);
  s.h.assign(n, 0.0);
  s.qx.assign(n, 0.0);
  s.qy.assign(n, 0.0);
  s.ks.assign(n, 0.0);
  s.twet.assign(n, 0.0);
  s.conc0.assign(n, 0.0);
  s.soil.assign(n, 0.0);
  s.ldry.assign(n, 0.0f);
  s.wall.assign(n, 0.0f);
  for (int icol = 1; icol <= NC; icol++) {
    for (int irow = 1; irow <= NR; irow++) {
      float zbp = (float)zb_raw[IX(irow, icol)];
      float zbp_corr;
      if (zbp == nodata || zbp == 0.0f) {
        float zbn = (float)zb_raw[IX(irow + 1, icol)], zbs = (float)zb_raw[IX(irow - 1, icol)];
        float zbe = (float)zb_raw[IX(irow, icol + 1)], zbw = (float)zb_raw[IX(irow, icol - 1)];
        int cnt = 0;
        zbp_corr = 0.0f;
        s.wall[IX(irow, icol)] = 1.0f;
        if (zbn != nodata && zbn != 0.0f && irow < NR) {
          zbp_corr += zbn;
          cnt++;
        }
        if (zbs != nodata && zbs != 0.0f && irow > 1) {
          zbp_corr += zbs;
          cnt++;
        }
        if (zbe != nodata && zbe != 0.0f && icol < NC) {
          zbp_corr += zbe;
          cnt++;
        }
        if (zbw != nodata && zbw != 0.0f && icol > 1) {
          zbp_corr += zbw;
          cnt++;
        }
        if (zbp_corr == 0.0f) zbp_corr = zbp;
        else zbp_corr /= cnt;
      } else {
        zbp_corr = std::fabs(zbp);
      }
      s.zb[IX(irow, icol)] = zbp_corr;
      s.ks[IX(irow, icol)] = ks_input;
    }
  }
  const int NR1 = NR + 1, NC1 = NC + 1;
  std::vector<double> zbs1(mr, 0.0);
  for (int irow = 0; irow <= NR1; irow++) {
    zbs1[irow] = s.zb[IX(irow, 1)];
    s.zb[IX(irow, 0)] = s.zb[IX(irow, 1)];
    s.zb[IX(irow, NC1)] = s.zb[IX(irow, NC)];
  }
  for (int icol = 0; icol <= NC1; icol++) {
    s.zb[IX(0, icol)] = s.zb[IX(1, icol)];
    s.zb[IX(NR1, icol)] = s.zb[IX(NR, icol)];
  }
  s.zb[IX(0, NC1)] = s.zb[IX(1, NC)];
  s.zb[IX(NR1, NC1)] = s.zb[IX(NR, NC)];
  for (int icol = 1; icol <= NC; icol++) {
    double zbsw = zbs1[1];
    int icol1 = icol + 1;
    double zbnw = s.zb[IX(1, icol1)];
    zbs1[1] = zbnw;
    for (int irow = 1; irow <= NR; irow++) {
      int irow1 = irow + 1;
      double zbse = zbs1[irow1];
      double zbne = s.zb[IX(irow1, icol1)];
      unsigned a = 0;
      double zbsum = 0;
      if (std::fabs(zbsw) != 99999) {
        zbsum = zbsum + zbsw;
        a = a + 1;
      }
      if (std::fabs(zbse) != 99999) {
        zbsum = zbsum + zbse;
        a = a + 1;
      }
      if (std::fabs(zbnw) != 99999) {
        zbsum = zbsum + zbnw;
        a = a + 1;
      }
      if (std::fabs(zbne) != 99999) {
        zbsum = zbsum + zbne;
        a = a + 1;
      }
      s.zb[IX(irow, icol)] = (zbsum) / a;
      zbs1[irow1] = zbne;
      zbsw = zbse;
      zbnw = zbne;
    }
  }
  for (int icol = 1; icol <= NC; icol++)
    for (int irow = 1; irow <= NR; irow++) {
      s.z[IX(irow, icol)] = s.zb[IX(irow, icol)];
      s.ldry[IX(irow, icol)] = 1.0f;
      s.conc0[IX(irow, icol)] = ade ? 0.0 : -1.0;
    }
}

// initiate.cpp:192-228: ghost ring of zb, z, h (run after the interior
// state, including a restart, is in place).
void ghost_ring(int NR, int NC, InitState& s) {
  const size_t mr = (size_t)NR + 2;
  auto IX = [mr](long r, long c) { return (size_t)c * mr + (size_t)r; };
  const int NR1 = NR + 1, NC1 = NC + 1;
  for (int icol = 0; icol <= NC1; icol++) {
    s.zb[IX(0, icol)] = 1.5 * s.zb[IX(1, icol)] - .5 * s.zb[IX(2, icol)];
    s.zb[IX(NR1, icol)] = 1.5 * s.zb[IX(NR, icol)] - .5 * s.zb[IX(NR - 1, icol)];
    s.z[IX(0, icol)] = 1.5 * s.z[IX(1, icol)] - .5 * s.z[IX(2, icol)];
    s.z[IX(NR1, icol)] = 1.5 * s.z[IX(NR, icol)] - .5 * s.z[IX(NR - 1, icol)];
    s.h[IX(0, icol)] = std::fmax(0.0, s.z[IX(0, icol)] - s.zb[IX(0, icol)]);
    s.h[IX(NR1, icol)] = std::fmax(0.0, s.z[IX(NR1, icol)] - s.zb[IX(NR1, icol)]);
    s.qx[IX(0, icol)] = 0.0;
    s.qy[IX(NR1, icol)] = 0.0;
  }
  for (int irow = 0; irow <= NR1; irow++) {
    s.zb[IX(irow, 0)] = 1.5 * s.zb[IX(irow, 1)] - .5 * s.zb[IX(irow, 2)];
    s.zb[IX(irow, NC1)] = 1.5 * s.zb[IX(irow, NC)] - .5 * s.zb[IX(irow, NC - 1)];
    s.z[IX(irow, 0)] = 1.5 * s.z[IX(irow, 1)] - .5 * s.z[IX(irow, 2)];
    s.z[IX(irow, NC1)] = 1.5 * s.z[IX(irow, NC)] - .5 * s.z[IX(irow, NC - 1)];
    s.h[IX(irow, 0)] = std::fmax(0.0, s.z[IX(irow, 0)] - s.zb[IX(irow, 0)]);
    s.h[IX(irow, NC1)] = std::fmax(0.0, s.z[IX(irow, NC1)] - s.zb[IX(irow, NC1)]);
    s.qx[IX(irow, 0)] = 0.0;
    s.qy[IX(irow, NC1)] = 0.0;
  }
}

// Newest Results/<t>.txt (what findLastStep of common.cpp:69-106 intends:
// the largest integer file stem in the folder).
long long last_results_time(const std::string& folder) {
  long long best = 0;
  DIR* dir = opendir(folder.c_str());
  if (!dir) return 0;
  while (dirent* e = readdir(dir)) {
    const char* nm = e->d_name;
    if (!isdigit((unsigned char)nm[0])) continue;
    long long v = atoll(nm);
    if (v > best) best = v;
  }
  closedir(dir);
  return best;
}

int upload_state(fx_ctx* c, const InitState& s) {
  int rc;
  if ((rc = fx_upload(c, "zb", s.zb.data()))) return rc;
  if ((rc = fx_upload(c, "z", s.z.data()))) return rc;
  if ((rc = fx_upload(c, "h", s.h.data()))) return rc;
  if ((rc = fx_upload(c, "qx", s.qx.data()))) return rc;
  if ((rc = fx_upload(c, "qy", s.qy.data()))) return rc;
  if ((rc = fx_upload(c, "twet", s.twet.data()))) return rc;
  for (int k = 0; k < c->g.nchem; ++k) {
    std::string nm = k == 0 ? "conc" : "conc" + std::to_string(k);
    if ((rc = fx_upload(c, nm.c_str(), s.conc0.data()))) return rc;
  }
  return fx_upload_flags(c, s.ldry.data(), s.wall.data());
}

// Appends v as printf's "%.17g" writes it (std::to_chars with the general
// format and precision 17 is specified to give the same characters).
inline void put17(std::string& out, double v) {
  char buf[40];
  const auto r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::general, 17);
  out.append(buf, r.ptr);
}

// One Results row (write_results.cpp:48-80): irow, icol, X, Y, z, z - zb,
// ux, uy, qx * dxy, qy * dxy, us, conc, soil_mass, fe_1, fn_1, twet, where
// ux, uy and us are 0 (never computed by the reference).
inline void put_row(std::string& out, int irow, int icol, int dxy, double xll, double yll, const double* v9) {
  const double row[16] = {(double)irow, (double)icol,
                          (double)((unsigned long)icol * (unsigned long)dxy) + xll,
                          (double)((unsigned long)irow * (unsigned long)dxy) + yll,
                          v9[0], v9[1], 0.0, 0.0, v9[2], v9[3], 0.0, v9[4], v9[5], v9[6], v9[7], v9[8]};
  for (int k = 0; k < 16; ++k) {
    put17(out, row[k]);
    out += (k < 15) ? ',' : '\n';
  }
}

const char* const kResultsHeader =
    "irow [-],icol [-],Xcoord,Ycoord,z [m],h [m],ux [m/s],uy [m/s],qx * dxy [m3/sec],"
    "qy * dxy [m3/sec],us [m/s],conc_SW [mg/l],soil_mass [g],fe_1 [m2/s],fn_1 [m2/s],"
    "twetimetracer [sec]\n";

// Rows as the device packs them (fx_results.cu): irow, icol, then
// FX_RES_NVAL columns of `n` values.
struct PackedRows {
  const int* irow;
  const int* icol;
  const double* v[FX_RES_NVAL];
  long long n;
};

PackedRows unpack(const void* buf, long long n) {
  PackedRows r;
  const char* p = (const char*)buf;
  r.irow = (const int*)p;
  r.icol = (const int*)(p + 4 * n);
  for (int k = 0; k < FX_RES_NVAL; ++k) r.v[k] = (const double*)(p + 8 * n + 8 * n * k);
  r.n = n;
  return r;
}

// Writes a Results file from packed rows: the text of blocks of rows is
// formatted by several threads, then written in order. With no row the
// reference still writes one row of zeros (write_results.cpp:309-310 keeps
// span(0, max(0, a-1))).
int write_packed(const std::string& path, const PackedRows& r, int dxy, double xll, double yll,
                 std::string& err) {
  FILE* fp = fopen(path.c_str(), "w");
  if (!fp) {
    err = "cannot write " + path;
    return FX_ERR_IO;
  }
  fputs(kResultsHeader, fp);
  if (r.n == 0) {
    for (int k = 0; k < 16; ++k) fputs(k < 15 ? "0," : "0\n", fp);
  } else {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const long long per = 16384;  // rows per thread and block
    const int nt = (int)std::min<long long>(hw, (r.n + per - 1) / per);
    std::vector<std::string> text(nt);
    for (long long base = 0; base < r.n; base += per * nt) {
      auto work = [&](int t) {
        std::string& out = text[t];
        out.clear();
        const long long a = base + per * t, b = std::min(r.n, a + per);
        double v9[FX_RES_NVAL];
        for (long long i = a; i < b; ++i) {
          for (int k = 0; k < FX_RES_NVAL; ++k) v9[k] = r.v[k][i];
          put_row(out, r.irow[i], r.icol[i], dxy, xll, yll, v9);
        }
      };
      std::vector<std::thread> th;
      for (int t = 1; t < nt; ++t) th.emplace_back(work, t);
      work(0);
      for (auto& x : th) x.join();
      for (int t = 0; t < nt; ++t) fwrite(text[t].data(), 1, text[t].size(), fp);
    }
  }
  if (fclose(fp) != 0) {
    err = "cannot write " + path;
    return FX_ERR_IO;
  }
  return FX_OK;
}

}  // namespace

// Results writer state of a context. Each file goes through one of two
// slots: the rows are compacted on the context's stream, copied to the
// slot's pinned buffer on a copy stream, and formatted and written by the
// slot's thread while the context keeps stepping.
struct fx_results_state {
  struct Slot {
    std::thread th;
    void* host = nullptr;  // pinned
    size_t cap = 0;
    cudaEvent_t copied = nullptr;
    int rc = FX_OK;
    std::string err;
  };
  Slot slot[2];
  int next = 0;
  cudaStream_t copy = nullptr;
  unsigned* counts = nullptr;   // device, nc
  long long* offs = nullptr;    // device, nc + 1
  void* rows = nullptr;         // device packed rows
  size_t rows_cap = 0;
  long long* total_host = nullptr;  // pinned
  cudaEvent_t rows_free = nullptr;  // the last copy out of `rows` is done
};

namespace {

int res_cuda(fx_ctx* c, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return FX_OK;
  return fx_fail(c, FX_ERR_CUDA, "%s failed: %s", what, cudaGetErrorString(e));
}

// Joins the slot's writer thread; returns its outcome.
int res_join(fx_ctx* c, fx_results_state::Slot& sl) {
  if (sl.th.joinable()) sl.th.join();
  const int rc = sl.rc;
  if (rc) fx_fail(c, rc, "%s", sl.err.c_str());
  sl.rc = FX_OK;
  sl.err.clear();
  return rc;
}

int res_init(fx_ctx* c) {
  if (c->res) return FX_OK;
  auto* r = new fx_results_state();
  c->res = r;
  int rc;
  if ((rc = res_cuda(c, cudaStreamCreateWithFlags(&r->copy, cudaStreamNonBlocking), "cudaStreamCreate")) ||
      (rc = res_cuda(c, cudaMalloc((void**)&r->counts, sizeof(unsigned) * (size_t)c->d.nc), "cudaMalloc")) ||
      (rc = res_cuda(c, cudaMalloc((void**)&r->offs, sizeof(long long) * ((size_t)c->d.nc + 1)), "cudaMalloc")) ||
      (rc = res_cuda(c, cudaMallocHost((void**)&r->total_host, sizeof(long long)), "cudaMallocHost")) ||
      (rc = res_cuda(c, cudaEventCreateWithFlags(&r->rows_free, cudaEventDisableTiming), "cudaEventCreate")))
    return rc;
  for (auto& sl : r->slot)
    if ((rc = res_cuda(c, cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming), "cudaEventCreate")))
      return rc;
  return FX_OK;
}

}  // namespace

void fx_results_release(fx_ctx* c) {
  if (!c || !c->res) return;
  fx_results_state* r = c->res;
  for (auto& sl : r->slot) {
    if (sl.th.joinable()) sl.th.join();
    if (sl.copied) cudaEventDestroy(sl.copied);
    if (sl.host) cudaFreeHost(sl.host);
  }
  if (r->copy) {
    cudaStreamSynchronize(r->copy);
    cudaStreamDestroy(r->copy);
  }
  if (r->rows_free) cudaEventDestroy(r->rows_free);
  if (r->rows) {
    cudaFree(r->rows);
    c->bytes -= (long long)r->rows_cap;
  }
  if (r->counts) cudaFree(r->counts);
  if (r->offs) cudaFree(r->offs);
  if (r->total_host) cudaFreeHost(r->total_host);
  delete r;
  c->res = nullptr;
}

extern "C" {

// read_geo's wall step and initiation's zero state from a raw DEM grid (the
// float DEM values in GlobVar layout, ghost ring 0), then upload and prepare.
int fx_initiate(fx_ctx* c, const double* zb_raw) {
  if (!c || !zb_raw) return fx_fail(c, FX_ERR_ARG, "fx_initiate: null argument");
  InitState s;
  initiate_bed(c->g.nrows, c->g.ncols, c->g.nodata, c->p.ks, c->p.ade != 0, zb_raw, s);
  ghost_ring(c->g.nrows, c->g.ncols, s);
  int rc = upload_state(c, s);
  if (rc) return rc;
  return fx_prepare(c);
}

// Host part of the start-up: everything fx_open_modset does before it
// touches the GPU. Call once with all buffers NULL to learn the sizes (g, p),
// then again with buffers of (nrows+2)*(ncols+2) elements (table: 3*2000).
int fx_load_modset(const char* modset_path, fx_grid* g_out, fx_params* p_out, double* zb, double* z,
                   double* h, double* qx, double* qy, double* twet, double* conc, double* soil_mass,
                   float* ldry, float* wall, float* table_2000x3, int* has_meteo) {
  if (!modset_path || !g_out || !p_out) return fx_fail(nullptr, FX_ERR_ARG, "fx_load_modset: null argument");
  Modset m;
  std::string err;
  int rc = read_modset(modset_path, m, err);
  if (rc) return fx_fail(nullptr, rc, "%s", err.c_str());
  Dem dm;
  if ((rc = read_dem(m.dem_file, dm, err))) return fx_fail(nullptr, rc, "%s", err.c_str());
  // forcing table (read_functions.cpp:237-282)
  std::vector<float> tab(3 * FX_METEO_ROWS, 0.0f);
  double tlast = 0.0;
  if (m.has_meteo) {
    bool ok = false;
    auto rows = read_csv_numbers(m.meteo_file, &ok);
    if (!ok) return fx_fail(nullptr, FX_ERR_IO, "cannot open METEO_FILE %s", m.meteo_file.c_str());
    if (rows.size() > (size_t)FX_METEO_ROWS)
      return fx_fail(nullptr, FX_ERR_ARG, "METEO_FILE has more than %d rows", FX_METEO_ROWS - 1);
    for (size_t a = 1; a < rows.size(); ++a) {
      for (int col = 0; col < 3; ++col)
        tab[(size_t)col * FX_METEO_ROWS + a] = (float)(col < (int)rows[a].size() ? rows[a][col] : 0.0);
      tlast = rows[a].empty() ? 0.0 : rows[a][0];
    }
  }
  fx_grid g{};
  g.nrows = dm.nrows;
  g.ncols = dm.ncols;
  g.dxy = dm.dxy;
  g.nchem = 1;
  g.nodata = dm.nodata;
  g.xll = dm.xll;
  g.yll = dm.yll;
  fx_params p{};
  p.hdry = m.ks;  // ks(1,1) (main.cpp:259)
  p.ks = m.ks;
  int ntim = (int)(float)tlast;  // float read_meteo -> int (main.cpp:74,181)
  if (m.has_inflow) {  // ntim = max(ntim_meteo, ntim_inflow) (main.cpp:184-192)
    std::vector<float> itab;
    double tin = 0.0;
    int irow = 0, icol = 0;
    if ((rc = read_inflow_table(m, itab, &tin, err)) ||
        (rc = inflow_cell(m, dm.xll, dm.yll, dm.dxy, dm.nrows, dm.ncols, &irow, &icol, err)))
      return fx_fail(nullptr, rc, "%s", err.c_str());
    ntim = std::max(ntim, (int)(float)tin);
  }
  p.ntim = (double)ntim;
  p.print_step = (double)m.print_step;
  p.h_min_print = (double)m.h_min_print;
  p.ade = m.ade ? 1 : 0;
  p.volrat_mode = 0;
  p.d_coef[0] = m.d_coef;
  p.wintra = (m.wintra && m.ade) ? 1 : 0;  // main.cpp:209-213
  p.soil_release_rate = m.soil_release_rate;
  long long timstart = 0;
  if (m.restart) timstart = last_results_time(m.output_folder);
  p.tim = 0.0;  // GlobVar::tim is never assigned before the loop (main.cpp:271)
  p.print_next = (double)(unsigned)(timstart + (long long)m.print_step);
  *g_out = g;
  *p_out = p;
  if (has_meteo) *has_meteo = m.has_meteo ? 1 : 0;
  if (!zb) return FX_OK;
  InitState s;
  initiate_bed(g.nrows, g.ncols, g.nodata, p.ks, m.ade, dm.zb_raw.data(), s);
  if (m.restart) {
    // initiate.cpp:115-158: rows of the newest Results file, columns
    // irow, icol, X, Y, z, h, ux, uy, qx, qy, us, conc, soil_mass, fe_1,
    // fn_1, twet (qx and qy are read back as written, i.e. times dxy).
    std::string fn = m.output_folder + "/" + std::to_string(timstart) + ".txt";
    bool ok = false;
    auto rows = read_csv_numbers(fn, &ok);
    if (ok) {
      const size_t mr = (size_t)g.nrows + 2;
      // initiate.cpp:93-107: the background soil mass where the bed is not
      // 99999, before the file's rows
      for (int icol = 1; icol <= g.ncols; icol++)
        for (int irow = 1; irow <= g.nrows; irow++) {
          const size_t i = (size_t)icol * mr + (size_t)irow;
          if (std::fabs(s.zb[i]) != 99999) s.soil[i] = m.soil_conc_bckgrd;
        }
      for (size_t a = 1; a < rows.size(); ++a) {
        const auto& r = rows[a];
        if (r.size() < 16) continue;
        long irow = (long)r[0], icol = (long)r[1];
        if (irow < 0 || irow > g.nrows + 1 || icol < 0 || icol > g.ncols + 1) continue;
        size_t i = (size_t)icol * mr + (size_t)irow;
        s.z[i] = r[4];
        s.h[i] = r[5];
        s.qx[i] = r[8];
        s.qy[i] = r[9];
        s.conc0[i] = m.ade ? std::fmax(r[11], 0.0) : -1.0;
        s.soil[i] = r[12];
        s.twet[i] = r[15];
        s.ldry[i] = 0.0f;
      }
    }
  }
  ghost_ring(g.nrows, g.ncols, s);
  const size_t n = ((size_t)g.nrows + 2) * ((size_t)g.ncols + 2);
  std::copy(s.zb.begin(), s.zb.end(), zb);
  if (z) std::copy(s.z.begin(), s.z.end(), z);
  if (h) std::copy(s.h.begin(), s.h.end(), h);
  if (qx) std::copy(s.qx.begin(), s.qx.end(), qx);
  if (qy) std::copy(s.qy.begin(), s.qy.end(), qy);
  if (twet) std::copy(s.twet.begin(), s.twet.end(), twet);
  if (conc) std::copy(s.conc0.begin(), s.conc0.end(), conc);
  if (soil_mass) std::copy(s.soil.begin(), s.soil.end(), soil_mass);
  if (ldry) std::copy(s.ldry.begin(), s.ldry.end(), ldry);
  if (wall) std::copy(s.wall.begin(), s.wall.end(), wall);
  if (table_2000x3) std::copy(tab.begin(), tab.end(), table_2000x3);
  (void)n;
  return FX_OK;
}

int fx_open_modset(const char* modset_path, fx_ctx** out) {
  if (!modset_path || !out) return fx_fail(nullptr, FX_ERR_ARG, "fx_open_modset: null argument");
  *out = nullptr;
  fx_grid g{};
  fx_params p{};
  int rc = fx_load_modset(modset_path, &g, &p, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                          nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
  if (rc) return rc;
  const size_t n = ((size_t)g.nrows + 2) * ((size_t)g.ncols + 2);
  std::vector<double> zb(n), z(n), h(n), qx(n), qy(n), tw(n), cc(n), soil(n);
  std::vector<float> ldry(n), wall(n), tab(3 * FX_METEO_ROWS);
  int has_meteo = 0;
  rc = fx_load_modset(modset_path, &g, &p, zb.data(), z.data(), h.data(), qx.data(), qy.data(), tw.data(),
                      cc.data(), soil.data(), ldry.data(), wall.data(), tab.data(), &has_meteo);
  if (rc) return rc;
  Modset m;
  std::string err;
  read_modset(modset_path, m, err);
  fx_ctx* c = nullptr;
  if ((rc = fx_create(&g, &p, &c))) return rc;
  c->output_folder = m.output_folder;
  mkdir(m.output_folder.c_str(), 0700);  // check_mkdir (common.cpp:393-405)
  if ((rc = fx_upload(c, "zb", zb.data())) || (rc = fx_upload(c, "z", z.data())) ||
      (rc = fx_upload(c, "h", h.data())) || (rc = fx_upload(c, "qx", qx.data())) ||
      (rc = fx_upload(c, "qy", qy.data())) || (rc = fx_upload(c, "twet", tw.data())) ||
      (rc = fx_upload(c, "conc", cc.data())) || (rc = fx_upload_flags(c, ldry.data(), wall.data())) ||
      (rc = fx_set_forcing(c, tab.data(), has_meteo)) ||
      ((p.wintra || std::any_of(soil.begin(), soil.end(), [](double v) { return v != 0.0; })) &&
       (rc = fx_upload(c, "soil_mass", soil.data())))) {
    std::string e = c->err;
    fx_destroy(c);
    return fx_fail(nullptr, rc, "%s", e.c_str());
  }
  if (m.has_inflow) {
    std::vector<float> itab;
    double tin = 0.0;
    int irow = 0, icol = 0;
    if ((rc = read_inflow_table(m, itab, &tin, err)) ||
        (rc = inflow_cell(m, g.xll, g.yll, g.dxy, g.nrows, g.ncols, &irow, &icol, err))) {
      fx_destroy(c);
      return fx_fail(nullptr, rc, "%s", err.c_str());
    }
    if ((rc = fx_set_inflow(c, itab.data(), irow, icol))) {
      std::string e = c->err;
      fx_destroy(c);
      return fx_fail(nullptr, rc, "%s", e.c_str());
    }
  }
  if ((rc = fx_prepare(c))) {
    std::string e = c->err;
    fx_destroy(c);
    return fx_fail(nullptr, rc, "%s", e.c_str());
  }
  *out = c;
  return FX_OK;
}

int fx_write_results_host(const char* path, int nrows, int ncols, int dxy, double xll, double yll,
                          double h_min_print, const double* z, const double* zb, const double* h,
                          const double* qx, const double* qy, const double* conc,
                          const double* soil_mass, const double* fe1, const double* fn1,
                          const double* twet) {
  if (!path || !z || !zb || !h || !qx || !qy || !conc || !fe1 || !fn1 || !twet)
    return fx_fail(nullptr, FX_ERR_ARG, "fx_write_results_host: null argument");
  // write_results.cpp:44-80: the selected cells (zb != 0, h > H_MIN_TO_PRINT)
  // in column-major order, packed as the device packs them
  const size_t mr = (size_t)nrows + 2;
  const double dx = (double)dxy;
  std::vector<int> ir, ic;
  std::vector<double> vals[FX_RES_NVAL];
  for (int icol = 1; icol <= ncols; icol++) {
    for (int irow = 1; irow <= nrows; irow++) {
      const size_t i = (size_t)icol * mr + (size_t)irow;
      if (zb[i] != 0.0 && h[i] > h_min_print) {
        const double v9[FX_RES_NVAL] = {z[i], z[i] - zb[i], qx[i] * dx, qy[i] * dx, conc[i],
                                        soil_mass ? soil_mass[i] : 0.0, fe1[i], fn1[i], twet[i]};
        ir.push_back(irow);
        ic.push_back(icol);
        for (int k = 0; k < FX_RES_NVAL; ++k) vals[k].push_back(v9[k]);
      }
    }
  }
  PackedRows r;
  r.irow = ir.data();
  r.icol = ic.data();
  for (int k = 0; k < FX_RES_NVAL; ++k) r.v[k] = vals[k].data();
  r.n = (long long)ir.size();
  std::string err;
  const int rc = write_packed(path, r, dxy, xll, yll, err);
  if (rc) return fx_fail(nullptr, rc, "%s", err.c_str());
  return FX_OK;
}

int fx_write_results_async(fx_ctx* c, const char* path) {
  if (!c) return FX_ERR_ARG;
  int rc;
  if (c->d.prec32 && c->z_pending && (rc = fx_prepare(c))) return rc;
  fx_status st;
  if ((rc = fx_get_status(c, &st))) return rc;
  std::string fn;
  if (path) fn = path;
  else fn = c->output_folder + "/" + std::to_string((long long)std::llround(st.print_next)) + ".txt";
  if ((rc = res_init(c)) || (rc = fx_sync_dev(c))) return rc;
  fx_results_state& r = *c->res;
  fx_results_state::Slot& sl = r.slot[r.next];
  r.next ^= 1;
  if ((rc = res_join(c, sl))) return rc;  // the slot's previous file
  // count and place the selected cells, then size the buffers
  fx_launch_results_count(c->d, c->h_min_print, r.counts, r.offs, c->stream);
  if ((rc = res_cuda(c, cudaMemcpyAsync(r.total_host, r.offs + c->d.nc, sizeof(long long),
                                        cudaMemcpyDeviceToHost, c->stream), "cudaMemcpyAsync")) ||
      (rc = res_cuda(c, cudaStreamSynchronize(c->stream), "results count")))
    return rc;
  const long long total = *r.total_host;
  const size_t bytes = (size_t)total * (8 + 8 * FX_RES_NVAL);
  if (bytes > r.rows_cap) {
    if ((rc = res_cuda(c, cudaEventSynchronize(r.rows_free), "cudaEventSynchronize"))) return rc;
    if (r.rows) {
      cudaFree(r.rows);
      c->bytes -= (long long)r.rows_cap;
      r.rows = nullptr;
      r.rows_cap = 0;
    }
    if ((rc = res_cuda(c, cudaMalloc(&r.rows, bytes), "cudaMalloc (Results rows)"))) return rc;
    r.rows_cap = bytes;
    c->bytes += (long long)bytes;
  }
  if (bytes > sl.cap) {
    if (sl.host) cudaFreeHost(sl.host);
    sl.host = nullptr;
    sl.cap = 0;
    if ((rc = res_cuda(c, cudaMallocHost(&sl.host, bytes), "cudaMallocHost (Results rows)"))) return rc;
    sl.cap = bytes;
  }
  // the previous file's copy out of the row buffer must be done first
  if ((rc = res_cuda(c, cudaStreamWaitEvent(c->stream, r.rows_free, 0), "cudaStreamWaitEvent"))) return rc;
  if (total > 0) fx_launch_results_write(c->d, c->h_min_print, r.offs, r.rows, total, c->stream);
  if ((rc = res_cuda(c, cudaGetLastError(), "results kernels")) ||
      (rc = res_cuda(c, cudaEventRecord(sl.copied, c->stream), "cudaEventRecord")) ||
      (rc = res_cuda(c, cudaStreamWaitEvent(r.copy, sl.copied, 0), "cudaStreamWaitEvent")))
    return rc;
  if (total > 0 && (rc = res_cuda(c, cudaMemcpyAsync(sl.host, r.rows, bytes, cudaMemcpyDeviceToHost, r.copy),
                                  "cudaMemcpyAsync (Results rows)")))
    return rc;
  if ((rc = res_cuda(c, cudaEventRecord(sl.copied, r.copy), "cudaEventRecord")) ||
      (rc = res_cuda(c, cudaEventRecord(r.rows_free, r.copy), "cudaEventRecord")))
    return rc;
  const int dxy = c->g.dxy;
  const double xll = c->g.xll, yll = c->g.yll;
  fx_results_state::Slot* sp = &sl;
  sl.th = std::thread([sp, fn, total, dxy, xll, yll]() {
    const cudaError_t e = cudaEventSynchronize(sp->copied);
    if (e != cudaSuccess) {
      sp->rc = FX_ERR_CUDA;
      sp->err = std::string("Results copy failed: ") + cudaGetErrorString(e);
      return;
    }
    sp->rc = write_packed(fn, unpack(sp->host, total), dxy, xll, yll, sp->err);
  });
  return FX_OK;
}

int fx_results_wait(fx_ctx* c) {
  if (!c) return FX_ERR_ARG;
  if (!c->res) return FX_OK;
  int first = FX_OK;
  for (auto& sl : c->res->slot) {
    const int rc = res_join(c, sl);
    if (rc && !first) first = rc;
  }
  return first;
}

int fx_write_results(fx_ctx* c, const char* path) {
  if (!c) return FX_ERR_ARG;
  int rc = fx_write_results_async(c, path);
  const int rw = fx_results_wait(c);
  return rc ? rc : rw;
}

int fx_run(const char* modset_path) {
  fx_ctx* c = nullptr;
  int rc = fx_open_modset(modset_path, &c);
  if (rc) return rc;
  fx_status st{};
  for (;;) {
    rc = fx_run_to_print(c, &st);
    if (rc) break;
    if (st.print_pending) {
      if ((rc = fx_write_results_async(c, nullptr))) break;  // written while the next steps run
      printf("Saved: '%lld.txt'\n", (long long)std::llround(st.print_next));
      if ((rc = fx_print_done(c))) break;
      continue;
    }
    if (st.finished) break;
  }
  const int rw = fx_results_wait(c);
  if (!rc) rc = rw;
  fx_destroy(c);
  return rc;
}


}  // extern "C"
