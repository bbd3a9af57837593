// qfiles.cpp -- readers and writers for Q's file formats.
//
//  * .inp and .fep: the keyword/section format of src/q6/prmfile.f90
//    (load 880-1000, split 1030-1065, *_by_key 108-330).
//  * .top: the list-directed topology format of src/q6/topo.f90:529-1079.
//  * .re: gfortran unformatted sequential records (md.f90:13650-13685 read,
//    md.f90:15452-15470 write).
//  * .en: put_ene records (src/q6/nrgy.f90:94-119).
//
// Fortran list-directed input is restated here: a READ starts at a new record,
// takes blank/comma separated values across as many records as it needs, and
// discards the rest of the last record it used.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <list>
#include <mutex>
#include <sstream>
#include <sys/stat.h>

#include "qsystem.hpp"

namespace qb {

namespace {

std::string upcase(std::string s) {
  for (auto &c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

// Fortran list-directed conversion of one token.
bool to_int(const std::string &tok, long &out) {
  if (tok.empty()) return false;
  char *end = nullptr;
  errno = 0;
  long v = std::strtol(tok.c_str(), &end, 10);
  if (*end != '\0' || errno) return false;
  out = v;
  return true;
}

bool to_real(std::string tok, double &out) {
  if (tok.empty()) return false;
  for (auto &c : tok)
    if (c == 'd' || c == 'D') c = 'e';
  char *end = nullptr;
  double v = std::strtod(tok.c_str(), &end);
  if (*end != '\0') return false;
  out = v;
  return true;
}

// Split a record into list-directed value tokens; stops at '/'.
// Expands r*c repeat counts.
void split_values(const std::string &line, std::vector<std::string> &toks, bool &slash) {
  slash = false;
  size_t i = 0, n = line.size();
  while (i < n) {
    while (i < n && (line[i] == ' ' || line[i] == '\t' || line[i] == ',' || line[i] == '\r')) i++;
    if (i >= n) break;
    if (line[i] == '/') { slash = true; return; }
    size_t j = i;
    if (line[i] == '\'' || line[i] == '"') {  // quoted string
      char q = line[i];
      j = i + 1;
      while (j < n && line[j] != q) j++;
      toks.push_back(line.substr(i + 1, j - i - 1));
      i = j + 1;
      continue;
    }
    while (j < n && line[j] != ' ' && line[j] != '\t' && line[j] != ',' && line[j] != '/' &&
           line[j] != '\r')
      j++;
    std::string t = line.substr(i, j - i);
    size_t star = t.find('*');
    long rep = 0;
    if (star != std::string::npos && star > 0 && to_int(t.substr(0, star), rep) && rep > 0) {
      std::string val = t.substr(star + 1);
      for (long r = 0; r < rep; r++) toks.push_back(val);
    } else {
      toks.push_back(t);
    }
    i = j;
  }
}

// Sequential reader over the records of a text file.
class Records {
 public:
  Records(const std::string &path) : path_(path) {
    std::ifstream f(path);
    if (!f) fail(QB_ERR_IO, "cannot open " + path);
    std::string l;
    while (std::getline(f, l)) {
      if (!l.empty() && l.back() == '\r') l.pop_back();
      lines_.push_back(l);
    }
  }
  bool eof() const { return cur_ >= lines_.size(); }
  size_t lineno() const { return cur_ + 1; }
  // read(u,'(a)') line
  std::string line() {
    if (eof()) err("unexpected end of file");
    return lines_[cur_++];
  }
  // read(u,*) with no items: skip one record
  void skip() { line(); }
  // read(u,*) v1..vn: list-directed values across records
  std::vector<std::string> values(size_t n) {
    std::vector<std::string> out;
    if (n == 0) return out;  // `if (n > 0) read(...)` in the reference: nothing consumed
    while (out.size() < n) {
      if (eof()) err("unexpected end of file reading values");
      bool slash = false;
      split_values(lines_[cur_++], out, slash);
      if (slash) break;
    }
    if (out.size() < n) err("too few values before '/'");
    out.resize(n);
    return out;
  }
  std::vector<long> ints(size_t n) {
    auto t = values(n);
    std::vector<long> r(n);
    for (size_t i = 0; i < n; i++)
      if (!to_int(t[i], r[i])) err("expected integer, got '" + t[i] + "'");
    return r;
  }
  std::vector<double> reals(size_t n) {
    auto t = values(n);
    std::vector<double> r(n);
    for (size_t i = 0; i < n; i++)
      if (!to_real(t[i], r[i])) err("expected real, got '" + t[i] + "'");
    return r;
  }
  long int1() { return ints(1)[0]; }
  // '(80i1)': n one-digit integers, 80 per record, blanks read as 0
  std::vector<int> digits(size_t n) {
    std::vector<int> r;
    r.reserve(n);
    while (r.size() < n) {
      std::string l = line();
      for (size_t c = 0; c < 80 && r.size() < n; c++) {
        char ch = c < l.size() ? l[c] : ' ';
        if (ch == ' ') r.push_back(0);
        else if (ch >= '0' && ch <= '9') r.push_back(ch - '0');
        else err("bad digit in (80i1) field");
      }
    }
    return r;
  }
  // '(80l1)': n logicals, 80 per record
  std::vector<unsigned char> logicals(size_t n) {
    std::vector<unsigned char> r;
    r.reserve(n);
    while (r.size() < n) {
      std::string l = line();
      for (size_t c = 0; c < 80 && r.size() < n; c++) {
        char ch = c < l.size() ? l[c] : ' ';
        r.push_back(ch == 'T' || ch == 't' ? 1 : 0);
      }
    }
    return r;
  }
  [[noreturn]] void err(const std::string &m) const {
    fail(QB_ERR_PARSE, path_ + ":" + std::to_string(cur_) + ": " + m);
  }

 private:
  std::string path_;
  std::vector<std::string> lines_;
  size_t cur_ = 0;
};

// Values of one record for an internal list-directed read with iostat: returns
// how many of the leading tokens convert.
std::vector<std::string> line_values(const std::string &line) {
  std::vector<std::string> t;
  bool slash;
  split_values(line, t, slash);
  return t;
}

// ------------------------------------------------------------ prmfile format

struct PrmSection {
  std::string name;
  std::vector<std::string> lines;
};

class PrmFile {
 public:
  explicit PrmFile(const std::string &path) {
    std::ifstream f(path);
    if (!f) fail(QB_ERR_IO, "cannot open " + path);
    std::string raw;
    while (std::getline(f, raw)) {
      if (!raw.empty() && raw.back() == '\r') raw.pop_back();
      size_t start = raw.find_first_not_of(" \t");
      if (start == std::string::npos) continue;
      char c0 = raw[start];
      if (c0 == '!' || c0 == '#' || c0 == '*') continue;
      if (c0 == '{') break;  // next title of a multi-title file
      if (c0 == '[') {
        size_t e = raw.find(']');
        if (e == std::string::npos || e <= start + 1) fail(QB_ERR_PARSE, "invalid section heading: " + raw);
        secs_.push_back({upcase(raw.substr(start + 1, e - start - 1)), {}});
        continue;
      }
      if (secs_.empty()) fail(QB_ERR_PARSE, path + ": data before first section");
      // strip a trailing comment (prmfile.f90:950-985)
      size_t cstart = std::string::npos;
      size_t last = raw.find_last_not_of(" \t");
      for (size_t p = start; p <= last; p++) {
        char c = raw[p];
        if (c == '!' || ((c == '#' || c == '*') && p > 0 && (raw[p - 1] == ' ' || raw[p - 1] == '\t'))) {
          cstart = p;
          break;
        }
      }
      std::string text;
      if (cstart != std::string::npos) {
        size_t ws = raw.find_last_of(" \t", cstart == 0 ? 0 : cstart - 1);
        size_t end = (ws == std::string::npos || ws < start) ? cstart : ws;
        text = raw.substr(start, end - start);
      } else {
        text = raw.substr(start, last - start + 1);
      }
      secs_.back().lines.push_back(text);
    }
  }
  const PrmSection *section(const std::string &name) const {
    std::string u = upcase(name);
    for (auto &s : secs_)
      if (s.name == u) return &s;
    return nullptr;
  }
  int count(const std::string &name) const {
    auto s = section(name);
    return s ? (int)s->lines.size() : 0;
  }

 private:
  std::vector<PrmSection> secs_;
};

// split (prmfile.f90:1030): key and first value token, or false.
bool prm_split(const std::string &line, std::string &key, std::string &val) {
  size_t a = line.find_first_not_of(" \t");
  if (a == std::string::npos) return false;
  size_t b = line.find_first_of(" \t", a);
  if (b == std::string::npos) return false;
  key = line.substr(a, b - a);
  size_t c = line.find_first_not_of(" \t", b + 1);
  if (c == std::string::npos) return false;
  size_t d = line.find_first_of(" \t!", c);
  val = line.substr(c, d == std::string::npos ? std::string::npos : d - c);
  return true;
}

// prm_get_*_by_key: the first line whose key matches exactly and whose value
// converts; the scan stops at the first line lacking a value.
bool get_real(const PrmSection *s, const std::string &key, double &out) {
  if (!s) return false;
  for (auto &l : s->lines) {
    std::string k, v;
    if (!prm_split(l, k, v)) return false;
    double d;
    auto t = line_values(v);
    if (k == key && !t.empty() && to_real(t[0], d)) { out = d; return true; }
  }
  return false;
}

bool get_int(const PrmSection *s, const std::string &key, int &out) {
  if (!s) return false;
  for (auto &l : s->lines) {
    std::string k, v;
    if (!prm_split(l, k, v)) return false;
    long d;
    auto t = line_values(v);
    if (k == key && !t.empty() && to_int(t[0], d)) { out = (int)d; return true; }
  }
  return false;
}

// prm_get_logical_by_key: 1 true, 0 false, -1 key absent, -2 invalid value
int get_logical(const PrmSection *s, const std::string &key) {
  if (!s) return -1;
  for (auto &l : s->lines) {
    std::string k, v;
    if (!prm_split(l, k, v)) return -1;
    if (k == key) {
      if (v == "on" || v == "ON" || v == "1") return 1;
      if (v == "off" || v == "OFF" || v == "0") return 0;
      return -2;
    }
  }
  return -1;
}

bool get_string(const PrmSection *s, const std::string &key, std::string &out) {
  if (!s) return false;
  std::string uk = upcase(key);
  for (auto &l : s->lines) {
    std::string k, v;
    if (!prm_split(l, k, v)) return false;
    if (upcase(k) == uk) { out = v; return true; }
  }
  return false;
}

bool logical_key(const PrmSection *s, const std::string &key, bool dflt, bool &out) {
  int r = get_logical(s, key);
  if (r == -1) { out = dflt; return true; }
  if (r == -2) return false;
  out = r == 1;
  return true;
}

std::string join_dir(const std::string &dir, const std::string &p) {
  if (p.empty() || p[0] == '/' || dir.empty()) return p;
  return dir + "/" + p;
}

}  // namespace

double fortran_pi() { return (double)(4.0f * std::atan(1.0f)); }
double fortran_deg2rad() { return fortran_pi() / 180.0; }

// ------------------------------------------------------------------- .inp

void read_inp(const std::string &path, RunInput &in) {
  PrmFile prm(path);
  in.inp_path = path;
  size_t slash = path.find_last_of('/');
  in.dir = slash == std::string::npos ? "" : path.substr(0, slash);
  std::vector<std::string> bad;

  // [PBC] (md.f90:2583-2656): periodic box, NVT or NPT (Monte Carlo volume moves)
  if (const PrmSection *pb = prm.section("PBC")) {
    in.box = true;
    if (!logical_key(pb, "rigid_box_center", false, in.rigid_box_center)) bad.push_back("rigid_box_center must be on or off");
    if (!logical_key(pb, "constant_pressure", false, in.constant_pressure)) bad.push_back("constant_pressure must be on or off");
    if (in.constant_pressure) {
      if (!get_real(pb, "max_volume_displ", in.max_vol_displ)) bad.push_back("maximum volume displacement not specified (section PBC)");
      if (!get_int(pb, "pressure_seed", in.pressure_seed)) in.pressure_seed = 3781;
      double p = 1.0;
      if (!get_real(pb, "pressure", p)) p = 1.0;
      in.pressure_bar = p;
      // bar to kcal/mol/A^3, the single-precision literal of md.f90:2619
      in.pressure = p * (double)1.43836e-5f;
    } else {
      for (auto &l : pb->lines) {
        std::string k, v;
        if (!prm_split(l, k, v)) break;
        if (k != "control_box") continue;
        auto t = line_values(l.substr(l.find(k) + k.size()));
        if (t.size() < 3 || !to_real(t[0], in.new_boxl[0]) || !to_real(t[1], in.new_boxl[1]) ||
            !to_real(t[2], in.new_boxl[2]))
          bad.push_back("control_box");
        in.control_box = true;
        break;
      }
    }
    // prm_get_logical_by_key without a default: absent keys leave the flags off
    bool b = false;
    if (get_logical(pb, "put_solvent_back_in_box") >= 0 && logical_key(pb, "put_solvent_back_in_box", false, b))
      in.put_solvent_back_in_box = b;
    if (get_logical(pb, "put_solute_back_in_box") >= 0 && logical_key(pb, "put_solute_back_in_box", false, b))
      in.put_solute_back_in_box = b;
  }
  const PrmSection *md = prm.section("MD");
  if (!md) fail(QB_ERR_UNSUPPORTED, path + ": no [MD] section (old-format input is not supported)");
  if (!get_int(md, "steps", in.nsteps)) bad.push_back("steps");
  if (!get_real(md, "stepsize", in.stepsize)) bad.push_back("stepsize");
  in.dt = 0.020462 * in.stepsize;
  if (!get_real(md, "temperature", in.Temp0)) bad.push_back("temperature");
  if (!get_real(md, "bath_coupling", in.tau_T)) in.tau_T = 10.0;
  in.tau_T = 0.020462 * in.tau_T;
  if (in.Temp0 <= 0) bad.push_back("temperature must be > 0");
  if (in.tau_T < in.dt) bad.push_back("bath_coupling < stepsize");
  if (!logical_key(md, "separate_scaling", false, in.separate_scaling)) bad.push_back("separate_scaling");
  if (!get_int(md, "random_seed", in.iseed)) in.iseed = 1;
  bool need_restart = false;
  if (get_real(md, "initial_temperature", in.Tmaxw)) {
    in.have_tmaxw = true;
  } else {
    in.iseed = 0;
    need_restart = true;
  }
  if (!logical_key(md, "shake_solvent", true, in.shake_solvent)) bad.push_back("shake_solvent");
  if (!logical_key(md, "shake_solute", false, in.shake_solute)) bad.push_back("shake_solute");
  if (!logical_key(md, "shake_hydrogens", false, in.shake_hydrogens)) bad.push_back("shake_hydrogens");
  bool b;
  if (logical_key(md, "lrf", false, b)) in.use_LRF = b;
  if (logical_key(md, "force_rms", false, b)) in.force_rms = b;

  // md.f90:2700 looks up 'cut-offs'; inputs spelling it 'cut_offs' get the defaults
  const PrmSection *co = prm.section("cut-offs");
  if (co) {
    // without LRF the section leaves RcLRF unset: zero, as the reference's
    // static variable (md.f90:2789), which the box checks see
    if (!in.use_LRF) in.RcLRF = 0.0;
    get_real(co, "solute_solute", in.Rcpp);
    get_real(co, "solvent_solvent", in.Rcww);
    get_real(co, "solute_solvent", in.Rcpw);
    get_real(co, "q_atom", in.Rcq);
    if (in.use_LRF) {
      get_real(co, "lrf", in.RcLRF);
      if (in.RcLRF < in.Rcpp || in.RcLRF < in.Rcpw || in.RcLRF < in.Rcww)
        bad.push_back("LRF cut-off smaller than solute or solvent cut-offs");
    }
  }
  const PrmSection *sp = prm.section("sphere");
  if (!sp) {
    in.fk_pshell = 10.0;
    in.rexcl_i = 0.85;
  } else {
    if (!get_real(sp, "shell_radius", in.rexcl_i)) in.rexcl_i = 0.85;
    else if (in.rexcl_i < 0) bad.push_back("shell_radius must be >= 0");
    if (!get_real(sp, "shell_force", in.fk_pshell)) in.fk_pshell = 10.0;
    if (!logical_key(sp, "exclude_bonded", false, in.exclude_bonded)) bad.push_back("exclude_bonded");
  }
  const PrmSection *sv = prm.section("solvent");
  if (!sv) sv = prm.section("water");
  if (!sv) {
    in.fk_wsphere = -1; in.Dwmz = -1; in.awmz = -1;
    in.wpol_restr = true; in.wpol_born = true; in.fkwpol = -1;
  } else {
    get_real(sv, "radius", in.rwat_in);
    if (!get_real(sv, "radial_force", in.fk_wsphere)) in.fk_wsphere = -1;
    logical_key(sv, "polarization", true, in.wpol_restr);
    logical_key(sv, "charge_correction", in.wpol_restr, in.wpol_born);
    if (in.wpol_born && !in.wpol_restr) bad.push_back("charge_correction requires polarization");
    if (!get_real(sv, "polarization_force", in.fkwpol)) in.fkwpol = -1;
    if (!get_real(sv, "morse_depth", in.Dwmz)) in.Dwmz = -1;
    if (!get_real(sv, "morse_width", in.awmz)) in.awmz = -1;
  }
  const PrmSection *iv = prm.section("intervals");
  if (!iv) {
    in.NBcycle = 10; in.iout_cycle = 10; in.itemp_cycle = 10; in.iene_cycle = 0; in.itrj_cycle = 0;
  } else {
    if (!get_int(iv, "non_bond", in.NBcycle)) in.NBcycle = 10;
    if (!get_int(iv, "output", in.iout_cycle)) in.iout_cycle = 10;
    if (!get_int(iv, "temperature", in.itemp_cycle)) in.itemp_cycle = 10;
    if (!get_int(iv, "energy", in.iene_cycle)) in.iene_cycle = 0;
    if (!get_int(iv, "trajectory", in.itrj_cycle)) in.itrj_cycle = 0;
    if (in.constant_pressure && !get_int(iv, "volume_change", in.ivolume_cycle)) in.ivolume_cycle = 10;
  }
  if (in.iout_cycle <= 0) in.iout_cycle = -999999999;
  if (in.itemp_cycle <= 0) in.itemp_cycle = -999999999;
  if (in.itrj_cycle <= 0) in.itrj_cycle = -999999999;
  if (in.iene_cycle <= 0) in.iene_cycle = -999999999;
  if (in.NBcycle <= 0) bad.push_back("non_bond interval must be > 0");

  const PrmSection *fl = prm.section("files");
  if (!fl) {
    bad.push_back("[files] section missing");
  } else {
    if (!get_string(fl, "topology", in.top_file)) bad.push_back("topology file");
    if (get_string(fl, "restart", in.restart_file)) in.restart = true;
    else if (need_restart) bad.push_back("restart file required without initial_temperature");
    if (!in.restart && in.iseed == 0) bad.push_back("random seed required to generate velocities");
    if (!get_string(fl, "final", in.xfin_file)) bad.push_back("final file");
    if (!get_string(fl, "trajectory", in.trj_file) && in.itrj_cycle > 0) bad.push_back("trajectory file");
    if (!get_string(fl, "energy", in.ene_file)) {
      if (in.iene_cycle > 0) bad.push_back("energy file");
    }
    if (!get_string(fl, "fep", in.fep_file)) in.fep_file = "";
    std::string r;
    if (get_string(fl, "restraint", r)) fail(QB_ERR_UNSUPPORTED, "[files] restraint (implicit restraint coordinates) is not supported");
  }
  in.lambdas.clear();
  if (auto la = prm.section("lambdas")) {
    for (auto &l : la->lines) {
      std::istringstream ss(l);
      std::string f;
      while (ss >> f) {
        double d;
        if (!to_real(f, d)) { bad.push_back("lambda value " + f); break; }
        in.lambdas.push_back(d);
      }
    }
  }
  if (in.lambdas.empty() && !in.fep_file.empty()) in.lambdas.push_back(1.0);
  if (!in.lambdas.empty() && in.fep_file.empty()) bad.push_back("lambdas given without FEP file");
  if ((int)in.lambdas.size() > QB_MAX_STATES) bad.push_back("too many states");

  if (auto s = prm.section("sequence_restraints")) {
    for (auto &l : s->lines) {
      auto t = line_values(l);
      SeqRestraint r{0, 0, 0, 0, 0};
      long li; double d;
      // read(text,*,end=,err=) stops at the first missing/invalid value
      if (t.size() > 0 && to_int(t[0], li)) { r.i = (int)li;
        if (t.size() > 1 && to_int(t[1], li)) { r.j = (int)li;
          if (t.size() > 2 && to_real(t[2], d)) { r.fk = d;
            if (t.size() > 3 && to_int(t[3], li)) { r.ih = (int)li;
              if (t.size() > 4 && to_int(t[4], li)) r.to_center = (int)li; } } } }
      r.i -= 1; r.j -= 1;
      in.rseq.push_back(r);
    }
  }
  if (auto s = prm.section("atom_restraints")) {
    for (auto &l : s->lines) {
      auto t = line_values(l);
      PosRestraint r{};
      long li; double d[7];
      bool ok = t.size() >= 8 && to_int(t[0], li);
      for (int k = 0; ok && k < 6; k++) ok = to_real(t[1 + k], d[k]);
      long ip = 0;
      ok = ok && to_int(t[7], ip);
      if (!ok) { bad.push_back("atom_restraints line: " + l); break; }
      r.i = (int)li - 1;
      for (int k = 0; k < 3; k++) { r.x[k] = d[k]; r.fk[k] = d[3 + k]; }
      r.ipsi = (int)ip;
      in.rpos.push_back(r);
    }
  }
  if (auto s = prm.section("distance_restraints")) {
    for (auto &l : s->lines) {
      auto t = line_values(l);
      if (l.find(':') != std::string::npos)
        fail(QB_ERR_UNSUPPORTED, "residue:atom distance restraints are not supported");
      DistRestraint r{};
      long a, bb, ip; double d1, d2, fk;
      if (t.size() < 6 || !to_int(t[0], a) || !to_int(t[1], bb) || !to_real(t[2], d1) ||
          !to_real(t[3], d2) || !to_real(t[4], fk) || !to_int(t[5], ip)) {
        bad.push_back("distance_restraints line: " + l);
        break;
      }
      r.i = (int)a - 1; r.j = (int)bb - 1; r.d1 = d1; r.d2 = d2; r.fk = fk; r.ipsi = (int)ip;
      in.rdis.push_back(r);
    }
  }
  if (auto s = prm.section("angle_restraints")) {
    for (auto &l : s->lines) {
      auto t = line_values(l);
      long a, bb, c, ip; double an, fk;
      if (t.size() < 6 || !to_int(t[0], a) || !to_int(t[1], bb) || !to_int(t[2], c) ||
          !to_real(t[3], an) || !to_real(t[4], fk) || !to_int(t[5], ip)) {
        bad.push_back("angle_restraints line: " + l);
        break;
      }
      in.rang.push_back({(int)a - 1, (int)bb - 1, (int)c - 1, an, fk, (int)ip});
    }
  }
  if (auto s = prm.section("wall_restraints")) {
    for (auto &l : s->lines) {
      auto t = line_values(l);
      long a, bb, ih; double dd, fk, am, dm;
      if (t.size() < 7 || !to_int(t[0], a) || !to_int(t[1], bb) || !to_real(t[2], dd) ||
          !to_real(t[3], fk) || !to_real(t[4], am) || !to_real(t[5], dm) || !to_int(t[6], ih)) {
        bad.push_back("wall_restraints line: " + l);
        break;
      }
      in.rwal.push_back({(int)a - 1, (int)bb - 1, dd, fk, am, dm, (int)ih});
    }
  }
  if (!bad.empty()) {
    std::string m = path + ": invalid data in input file:";
    for (auto &x : bad) m += " [" + x + "]";
    fail(QB_ERR_PARSE, m);
  }
  in.top_file = join_dir(in.dir, in.top_file);
  if (!in.fep_file.empty()) in.fep_file = join_dir(in.dir, in.fep_file);
  if (in.restart) in.restart_file = join_dir(in.dir, in.restart_file);
  in.xfin_file = join_dir(in.dir, in.xfin_file);
  if (!in.ene_file.empty()) in.ene_file = join_dir(in.dir, in.ene_file);
  if (!in.trj_file.empty()) in.trj_file = join_dir(in.dir, in.trj_file);
}

// --------------------------------------------------------------- topology

namespace {
void parse_topology(const std::string &path, Topology &t);

// Parsed topologies by file identity (path, size, modification time): a
// perturbation opens one .inp once per window and replica, and parsing the
// text topology dominated opening.  Entries are copied out, never shared.
struct TopologyCache {
  struct Entry {
    std::string path;
    long long size, mtime_ns;
    Topology top;
  };
  std::mutex mu;
  std::list<Entry> entries;   // most recent first
  static constexpr size_t kMax = 8;
};
TopologyCache g_topology_cache;
}  // namespace

void read_topology(const std::string &path, Topology &t) {
  struct stat st;
  if (stat(path.c_str(), &st) != 0) { parse_topology(path, t); return; }
  const long long size = (long long)st.st_size;
  const long long mtime = (long long)st.st_mtim.tv_sec * 1000000000LL + st.st_mtim.tv_nsec;
  {
    std::lock_guard<std::mutex> g(g_topology_cache.mu);
    for (auto it = g_topology_cache.entries.begin(); it != g_topology_cache.entries.end(); ++it)
      if (it->path == path && it->size == size && it->mtime_ns == mtime) {
        t = it->top;
        g_topology_cache.entries.splice(g_topology_cache.entries.begin(), g_topology_cache.entries, it);
        return;
      }
  }
  parse_topology(path, t);
  std::lock_guard<std::mutex> g(g_topology_cache.mu);
  g_topology_cache.entries.push_front({path, size, mtime, t});
  if (g_topology_cache.entries.size() > TopologyCache::kMax) g_topology_cache.entries.pop_back();
}

namespace {
void parse_topology(const std::string &path, Topology &t) {
  Records r(path);
  std::string title = r.line();
  t.ff_type = 1;
  if (trim(title) == "Q topology file") {
    for (;;) {
      std::string l = r.line();
      auto toks = line_values(l);
      if (toks.empty()) continue;
      std::string key = upcase(toks[0]);
      size_t kp = l.find(toks[0]);
      std::string rest = trim(l.substr(kp + toks[0].size()));
      if (key == "TITLE") t.title = rest;
      else if (key == "VERSION") to_real(line_values(rest).at(0), t.version);
      else if (key == "FF_TYPE") { long ff; if (to_int(line_values(rest).at(0), ff)) t.ff_type = (int)ff; }
      else if (key == "END") break;
    }
  } else {
    t.title = title;
    t.version = 2;
  }
  if (t.version < 4.15) fail(QB_ERR_PARSE, path + ": topology version < 4.15");

  // 2. atoms
  {
    std::string l = r.line();
    auto v = line_values(l);
    long a = 0, b = 0;
    if (v.empty() || !to_int(v[0], a)) r.err("number of atoms");
    t.nat_pro = (int)a;
    t.nat_solute = (v.size() > 1 && to_int(v[1], b)) ? (int)b : t.nat_pro;
  }
  int N = t.nat_pro;
  if (N <= 0) fail(QB_ERR_PARSE, path + ": zero atoms");
  int nwat = (N - t.nat_solute) / 3;
  t.xtop = r.reals(3 * (size_t)N);
  r.skip();
  {
    auto ia = r.ints(N);
    t.iac.resize(N);
    for (int i = 0; i < N; i++) t.iac[i] = (int)ia[i] - 1;
  }
  // 5. bonds
  auto count_pair = [&](int &total, int &solute) {
    std::string l = r.line();
    auto v = line_values(l);
    long a = 0, b = 0;
    if (v.empty() || !to_int(v[0], a)) r.err("count");
    total = (int)a;
    solute = (v.size() > 1 && to_int(v[1], b)) ? (int)b : total;
  };
  int nb, nbs;
  count_pair(nb, nbs);
  t.nbonds_solute = nbs;
  {
    auto v = r.ints(3 * (size_t)nb);
    t.bnd.resize(nb);
    for (int i = 0; i < nb; i++) t.bnd[i] = {(int)v[3 * i] - 1, (int)v[3 * i + 1] - 1, (int)v[3 * i + 2]};
  }
  int nbndcod = (int)r.int1();
  t.bond_fk.assign(nbndcod, 0.0);
  t.bond_b0.assign(nbndcod, 0.0);
  for (int i = 0; i < nbndcod; i++) {
    auto v = line_values(r.line());
    double fk, b0;
    if (v.size() >= 3 && to_real(v[1], fk) && to_real(v[2], b0)) { t.bond_fk[i] = fk; t.bond_b0[i] = b0; }
  }
  // 6. angles
  int na, nas;
  count_pair(na, nas);
  t.nangles_solute = nas;
  {
    auto v = r.ints(4 * (size_t)na);
    t.ang.resize(na);
    for (int i = 0; i < na; i++)
      t.ang[i] = {(int)v[4 * i] - 1, (int)v[4 * i + 1] - 1, (int)v[4 * i + 2] - 1, (int)v[4 * i + 3]};
  }
  int nangcod = (int)r.int1();
  t.ang_fk.assign(nangcod, 0.0);
  t.ang_th0.assign(nangcod, 0.0);
  t.ang_ureyfk.assign(nangcod, 0.0);
  t.ang_ureyr0.assign(nangcod, 0.0);
  // "code fk theta0 [ureyfk [ureyr0]]": the Urey-Bradley pair is optional
  // and stays zero when the line ends first (topo.f90:712-726)
  for (int i = 0; i < nangcod; i++) {
    auto v = line_values(r.line());
    double fk, a0;
    if (v.size() < 3 || !to_real(v[1], fk) || !to_real(v[2], a0)) r.err("angle parameters");
    t.ang_fk[i] = fk;
    t.ang_th0[i] = a0;
    if (v.size() > 3 && !to_real(v[3], t.ang_ureyfk[i])) r.err("angle parameters");
    if (v.size() > 4 && !to_real(v[4], t.ang_ureyr0[i])) r.err("angle parameters");
  }
  // 7. torsions
  int nt, nts;
  count_pair(nt, nts);
  t.ntors_solute = nts;
  {
    auto v = r.ints(5 * (size_t)nt);
    t.tor.resize(nt);
    for (int i = 0; i < nt; i++)
      t.tor[i] = {(int)v[5 * i] - 1, (int)v[5 * i + 1] - 1, (int)v[5 * i + 2] - 1, (int)v[5 * i + 3] - 1,
                  (int)v[5 * i + 4]};
  }
  int ntorcod = (int)r.int1();
  for (int i = 0; i < ntorcod; i++) {
    auto v = r.reals(5);
    t.tor_fk.push_back((float)v[1]);
    t.tor_rmult.push_back((float)v[2]);
    t.tor_deltor.push_back((float)v[3]);
    t.tor_paths.push_back((float)v[4]);
  }
  // 8. impropers
  int ni, nis;
  count_pair(ni, nis);
  t.nimps_solute = nis;
  {
    auto v = r.ints(5 * (size_t)ni);
    t.imp.resize(ni);
    for (int i = 0; i < ni; i++)
      t.imp[i] = {(int)v[5 * i] - 1, (int)v[5 * i + 1] - 1, (int)v[5 * i + 2] - 1, (int)v[5 * i + 3] - 1,
                  (int)v[5 * i + 4]};
  }
  int nimpcod;
  {
    auto v = line_values(r.line());
    long a = 0, b = 0;
    if (v.empty() || !to_int(v[0], a)) r.err("number of improper codes");
    nimpcod = (int)a;
    t.imp_type = (v.size() > 1 && to_int(v[1], b)) ? (int)b : 1;
  }
  for (int i = 0; i < nimpcod; i++) {
    auto v = r.reals(3);
    t.imp_fk.push_back((float)v[1]);
    t.imp_imp0.push_back((float)v[2]);
  }
  // 9. charges
  {
    auto v = line_values(r.line());
    long n2;
    if (!v.empty() && to_int(v[0], n2) && n2 != N) r.err("charge count differs from atom count");
    auto c = r.reals(N);
    t.crg.resize(N);
    for (int i = 0; i < N; i++) t.crg[i] = (float)c[i];
  }
  // 10. charge groups
  {
    auto v = line_values(r.line());
    long a = 0, b = 0, c = 1;
    if (v.empty() || !to_int(v[0], a)) r.err("number of charge groups");
    t.ncgp = (int)a;
    t.ncgp_solute = (v.size() > 1 && to_int(v[1], b)) ? (int)b : t.ncgp;
    t.iuse_switch_atom = (v.size() > 2 && to_int(v[2], c)) ? (int)c : 1;
  }
  t.cgp_iswitch.resize(t.ncgp);
  t.cgp_first.resize(t.ncgp);
  t.cgp_last.resize(t.ncgp);
  t.cgpatom.assign(N, 0);
  {
    int k = 0;
    for (int i = 0; i < t.ncgp; i++) {
      auto v = r.ints(2);
      int n = (int)v[0];
      t.cgp_iswitch[i] = (int)v[1] - 1;
      t.cgp_first[i] = k;
      t.cgp_last[i] = k + n - 1;
      if (k + n > N) r.err("charge group atoms exceed atom count");
      auto a = r.ints(n);
      for (int j = 0; j < n; j++) t.cgpatom[k + j] = (int)a[j] - 1;
      k += n;
    }
  }
  // 11. masses and LJ
  t.natyps = (int)r.int1();
  t.ivdw_rule = (int)r.int1();
  {
    auto v = line_values(r.line());
    double e14, cc;
    if (v.empty() || !to_real(v[0], e14)) r.err("el14 scale");
    t.el14_scale = e14;
    t.coulomb_constant = (v.size() > 1 && to_real(v[1], cc) && cc > 0) ? cc : 332.0;
  }
  t.iaclib.resize(t.natyps);
  r.skip();
  {
    auto m = r.reals(t.natyps);
    for (int i = 0; i < t.natyps; i++) t.iaclib[i].mass = m[i];
  }
  for (int j = 0; j < 3; j++) {
    r.skip();
    auto a = r.reals(t.natyps);
    r.skip();
    auto bb = r.reals(t.natyps);
    for (int i = 0; i < t.natyps; i++) { t.iaclib[i].avdw[j] = a[i]; t.iaclib[i].bvdw[j] = bb[i]; }
  }
  {
    int nlj2 = (int)r.int1();
    for (int i = 0; i < nlj2; i++) {
      auto v = r.ints(2);
      t.lj2.push_back({(int)v[0] - 1, (int)v[1] - 1});
    }
  }
  t.heavy.resize(N);
  for (int i = 0; i < N; i++) {
    if (t.iac[i] < 0 || t.iac[i] >= t.natyps) r.err("atom type out of range");
    t.heavy[i] = t.iaclib[t.iac[i]].mass < 4.0 ? 0 : 1;
  }
  // 12. 1-4 and exclusion lists
  auto bits = [&](std::vector<unsigned int> &out) {
    out.assign(t.nat_solute, 0u);
    if (t.nat_solute > 0) {
      auto d = r.digits((size_t)QB_NBR_RANGE * t.nat_solute);
      for (int j = 0; j < t.nat_solute; j++)
        for (int i = 0; i < QB_NBR_RANGE; i++)
          if (d[(size_t)j * QB_NBR_RANGE + i] == 1) out[j] |= 1u << i;
    }
  };
  r.int1();  // n14nbrs
  bits(t.list14);
  {
    int n = (int)r.int1();
    for (int i = 0; i < n; i++) {
      auto v = r.ints(2);
      t.list14long.push_back({(int)v[0] - 1, (int)v[1] - 1});
    }
  }
  r.int1();  // nexnbrs
  bits(t.listex);
  {
    int n = (int)r.int1();
    for (int i = 0; i < n; i++) {
      auto v = r.ints(2);
      t.listexlong.push_back({(int)v[0] - 1, (int)v[1] - 1});
    }
  }
  // residues and molecules
  {
    std::string l = r.line();
    if (trim(l).empty()) l = r.line();
    auto v = line_values(l);
    long a = 0, b = 0;
    if (v.empty() || !to_int(v[0], a)) r.err("number of residues");
    t.nres = (int)a;
    t.nres_solute = (v.size() > 1 && to_int(v[1], b)) ? (int)b : t.nres;
    if (t.nres > 0) {
      auto s = r.ints(t.nres);
      for (auto x : s) t.res_start.push_back((int)x - 1);
    }
    r.skip();
    for (int i = 0; i < (t.nres + 15) / 16; i++) {
      std::string nl = r.line();
      for (int j = 0; j < 16 && i * 16 + j < t.nres; j++)
        t.res_name.push_back(trim(nl.size() > (size_t)j * 5 ? nl.substr(j * 5, 4) : ""));
    }
  }
  t.nmol = (int)r.int1();
  if (t.nmol > 0) {
    auto s = r.ints(t.nmol);
    for (auto x : s) t.istart_mol.push_back((int)x - 1);
  }
  t.istart_mol.push_back(N);
  r.skip();
  for (int i = 0; i < (t.natyps + 7) / 8; i++) {
    std::string nl = r.line();
    for (int j = 0; j < 8 && i * 8 + j < t.natyps; j++)
      t.tac.push_back(trim(nl.size() > (size_t)j * 9 ? nl.substr(j * 9, 8) : ""));
  }
  r.skip();
  for (int i = 0; i < (t.natyps + 12) / 13; i++) r.skip();
  t.solvent_type = (int)r.int1();
  {
    std::string l = r.line();
    auto v = line_values(l);
    if (v.empty()) r.err("boundary line");
    if (v[0] == "PBC") {
      // periodic box (topo.f90:1027-1036): edge lengths and centre; no
      // excluded atoms, no restrained shell, nothing further in the file
      t.use_pbc = true;
      auto bl = r.reals(3);
      auto bc = r.reals(3);
      for (int k = 0; k < 3; k++) { t.boxlength[k] = bl[k]; t.boxcenter[k] = bc[k]; }
      t.excl.assign(N, 0);
      return;
    }
    t.use_pbc = false;
    double a, b, c;
    if (t.version < 5.01) {
      if (v.size() < 3 || !to_real(v[0], a) || !to_real(v[1], b) || !to_real(v[2], c)) r.err("sphere radii");
      t.rexcl_o = a; t.rwat = c;
    } else {
      if (v.size() < 2 || !to_real(v[0], a) || !to_real(v[1], b)) r.err("sphere radii");
      t.rexcl_o = a; t.rwat = b;
    }
    auto pc = r.reals(3);
    auto wc = r.reals(3);
    for (int k = 0; k < 3; k++) { t.xpcent[k] = pc[k]; t.xwcent[k] = wc[k]; }
    auto ne = r.ints(2);
    t.nexats = (int)ne[0];
    t.nexwat = (int)ne[1];
    t.excl = r.logicals(N);
  }
  (void)nwat;
}
}  // namespace

// -------------------------------------------------------------------- FEP

void read_fep_atoms(const std::string &path, const Topology &t, Fep &f, int nstates_inp) {
  PrmFile prm(path);
  const PrmSection *at = prm.section("atoms");
  if (!at) fail(QB_ERR_UNSUPPORTED, path + ": old-format FEP file (no [atoms] section) is not supported");
  const PrmSection *fep = prm.section("FEP");
  f.nstates = 1;
  f.offset = 0;
  if (fep) {
    int ns;
    if (get_int(fep, "states", ns)) f.nstates = ns;
    bool b;
    if (logical_key(fep, "qq_use_library_charges", false, b)) f.qq_use_library_charges = b;
    if (logical_key(fep, "softcore_use_max_potential", false, b)) f.softcore_use_max_potential = b;
    int off;
    std::string s;
    if (get_int(fep, "offset", off)) {
      if (off < 1 || off > t.nat_solute) fail(QB_ERR_PARSE, "invalid topology atom number offset");
      f.offset = off;
    } else if (get_string(fep, "offset_name", s) || get_int(fep, "offset_residue", off)) {
      fail(QB_ERR_UNSUPPORTED, "residue-based FEP offsets are not supported");
    }
  }
  if (f.nstates <= 0) fail(QB_ERR_PARSE, "number of states must be at least 1");
  (void)nstates_inp;
  int nlines = (int)at->lines.size();
  if (nlines == 0) { f.nqat = 0; return; }
  // case 1 (qatom.f90:338): "q-atom  topology-atom" integer pairs
  int maxq = 0;
  std::vector<std::pair<long, long>> pairs;
  for (auto &l : at->lines) {
    auto v = line_values(l);
    long a, b;
    if (v.size() < 2 || !to_int(v[0], a) || !to_int(v[1], b))
      fail(QB_ERR_UNSUPPORTED, "only numeric [atoms] entries are supported: " + l);
    pairs.push_back({a, b});
    maxq = std::max<int>(maxq, (int)a);
  }
  f.nqat = maxq;
  f.iqseq.assign(maxq, -1);
  for (auto &p : pairs) {
    long topno = p.second + f.offset;
    if (topno < 1 || topno > t.nat_solute || p.first < 1)
      fail(QB_ERR_PARSE, "invalid topology atom number for Q-atom");
    f.iqseq[p.first - 1] = (int)topno - 1;
  }
}

void read_fep(const std::string &path, const Topology &t, Fep &f) {
  PrmFile prm(path);
  const int S = f.nstates, nq = f.nqat;
  const double deg2rad = fortran_deg2rad();
  auto lines = [&](const char *name) -> const std::vector<std::string> & {
    static const std::vector<std::string> empty;
    auto s = prm.section(name);
    return s ? s->lines : empty;
  };
  auto bad = [&](const std::string &m) { fail(QB_ERR_PARSE, path + ": " + m); };
  // a periodic box needs the Q atoms' switching atom (qatom.f90:910-925)
  if (t.use_pbc) {
    const PrmSection *pb = prm.section("PBC");
    if (!pb) bad("section PBC is required when using periodic boundary");
    int sw = 0;
    if (!get_int(pb, "switching_atom", sw)) bad("switching atom could not be read");
    f.qswitch = sw - 1 + f.offset;
    if (f.qswitch < 0 || f.qswitch >= t.nat_pro) bad("switching_atom out of range");
  }
  // f.qcrg holds the library charges (get_fep md.f90:1495-1500)
  for (auto &l : lines("change_charges")) {
    auto v = line_values(l);
    long iq;
    if (v.size() < (size_t)(1 + S) || !to_int(v[0], iq) || iq < 1 || iq > nq || f.iqseq[iq - 1] < 0)
      bad("change_charges: " + l);
    for (int s = 0; s < S; s++) {
      double c;
      if (!to_real(v[1 + s], c)) bad("change_charges: " + l);
      f.qcrg[(iq - 1) * S + s] = (float)c;
    }
  }
  std::vector<std::string> tac;
  for (auto &l : lines("atom_types")) {
    auto v = line_values(l);
    if (v.size() < 8) bad("atom_types: " + l);
    tac.push_back(v[0]);
    for (int k = 0; k < 3; k++) {
      double a, b;
      if (!to_real(v[1 + 2 * k], a) || !to_real(v[2 + 2 * k], b)) bad("atom_types: " + l);
      f.qavdw.push_back(a);
      f.qbvdw.push_back(b);
    }
    double m;
    if (!to_real(v[7], m)) bad("atom_types mass: " + l);
    f.qmass.push_back(m);
  }
  f.nqlib = (int)tac.size();
  f.qtac = tac;
  f.qiac.assign((size_t)nq * S, 0);
  {
    auto &ca = lines("change_atoms");
    int maxe = 0;
    for (auto &l : ca) { auto v = line_values(l); long a; if (!v.empty() && to_int(v[0], a)) maxe = std::max<int>(maxe, (int)a); }
    if (maxe == 0) {
      f.qvdw_flag = false;
    } else if (maxe != nq || (int)ca.size() != nq) {
      bad("change_atoms must list every Q-atom");
    } else {
      f.qvdw_flag = true;
      for (auto &l : ca) {
        auto v = line_values(l);
        long iq;
        if (v.size() < (size_t)(1 + S) || !to_int(v[0], iq) || iq < 1 || iq > nq) bad("change_atoms: " + l);
        for (int s = 0; s < S; s++) {
          auto it = std::find(tac.begin(), tac.end(), v[1 + s]);
          if (it == tac.end()) bad("Q-atom type " + v[1 + s] + " has not been defined");
          f.qiac[(iq - 1) * S + s] = (int)(it - tac.begin());
        }
      }
    }
  }
  for (auto &l : lines("soft_pairs")) {
    auto v = line_values(l);
    long a, b;
    if (v.size() < 2 || !to_int(v[0], a) || !to_int(v[1], b) || a < 1 || a > nq || b < 1 || b > nq) bad("soft_pairs: " + l);
    f.soft_pairs.push_back({(int)a - 1, (int)b - 1});
  }
  for (auto &l : lines("el_scale")) {
    auto v = line_values(l);
    long a, b;
    if (v.size() < (size_t)(2 + S) || !to_int(v[0], a) || !to_int(v[1], b) || a < 1 || a > nq || b < 1 || b > nq)
      bad("el_scale: " + l);
    Fep::ElScale e{(int)a - 1, (int)b - 1, {}};
    for (int s = 0; s < S; s++) if (!to_real(v[2 + s], e.s[s])) bad("el_scale: " + l);
    f.el_scale.push_back(e);
  }
  for (auto &l : lines("excluded_pairs")) {
    auto v = line_values(l);
    long a, b;
    if (v.size() < (size_t)(2 + S) || !to_int(v[0], a) || !to_int(v[1], b)) bad("excluded_pairs: " + l);
    Fep::ExSpec e{(int)(a + f.offset) - 1, (int)(b + f.offset) - 1, {}};
    for (int s = 0; s < S; s++) {
      long fl;
      if (!to_int(v[2 + s], fl) || (fl != 0 && fl != 1)) bad("excluded_pairs flags: " + l);
      e.flag[s] = fl == 1;
    }
    f.exspec.push_back(e);
  }
  // bond types: Morse "Dmz amz r0" or harmonic "fk r0" (qatom.f90:1105-1130)
  {
    auto &bt = lines("bond_types");
    int maxe = 0;
    for (auto &l : bt) { auto v = line_values(l); long a; if (!v.empty() && to_int(v[0], a)) maxe = std::max<int>(maxe, (int)a); }
    f.qbondlib.assign(maxe, {0, 0, 0, 0});
    std::vector<char> seen(maxe, 0);
    for (auto &l : bt) {
      auto v = line_values(l);
      long j; double a, b, c;
      if (v.empty() || !to_int(v[0], j) || j < 1) bad("bond_types: " + l);
      if (v.size() >= 4 && to_real(v[1], a) && to_real(v[2], b) && to_real(v[3], c)) {
        f.qbondlib[j - 1] = {a, b, c, 0.0};
      } else if (v.size() >= 3 && to_real(v[1], a) && to_real(v[2], b)) {
        f.qbondlib[j - 1] = {0.0, 0.0, b, a};
      } else bad("bond_types: " + l);
      seen[j - 1] = 1;
    }
    for (auto &l : lines("change_bonds")) {
      auto v = line_values(l);
      long a, b;
      if (v.size() < (size_t)(2 + S) || !to_int(v[0], a) || !to_int(v[1], b)) bad("change_bonds: " + l);
      Fep::QBnd q{(int)(a + f.offset) - 1, (int)(b + f.offset) - 1, {}};
      for (int s = 0; s < S; s++) {
        long c;
        if (!to_int(v[2 + s], c)) bad("change_bonds: " + l);
        if (c > 0 && (c > maxe || !seen[c - 1])) bad("undefined Q-bond type in: " + l);
        q.cod[s] = (int)c;
      }
      f.qbnd.push_back(q);
    }
  }
  {
    auto &at = lines("angle_types");
    int maxe = 0;
    for (auto &l : at) { auto v = line_values(l); long a; if (!v.empty() && to_int(v[0], a)) maxe = std::max<int>(maxe, (int)a); }
    f.qanglib.assign(maxe, {0, 0, 0, 0});
    for (auto &l : at) {
      auto v = line_values(l);
      long j; double fk, a0, ufk = 0, ur0 = 0;
      if (v.size() < 3 || !to_int(v[0], j) || j < 1 || !to_real(v[1], fk) || !to_real(v[2], a0)) bad("angle_types: " + l);
      // optional Urey-Bradley force constant and 1-3 distance (qatom.f90:1213-1236)
      if ((v.size() > 3 && !to_real(v[3], ufk)) || (v.size() > 4 && !to_real(v[4], ur0))) bad("angle_types: " + l);
      f.qanglib[j - 1] = {fk, deg2rad * a0, ufk, ur0};
    }
    for (auto &l : lines("change_angles")) {
      auto v = line_values(l);
      long a, b, c;
      if (v.size() < (size_t)(3 + S) || !to_int(v[0], a) || !to_int(v[1], b) || !to_int(v[2], c)) bad("change_angles: " + l);
      Fep::QAng q{(int)(a + f.offset) - 1, (int)(b + f.offset) - 1, (int)(c + f.offset) - 1, {}};
      for (int s = 0; s < S; s++) {
        long cc;
        if (!to_int(v[3 + s], cc) || cc > maxe) bad("change_angles: " + l);
        q.cod[s] = (int)cc;
      }
      f.qang.push_back(q);
    }
  }
  auto tors = [&](const char *types, const char *changes, std::vector<double> &fk, std::vector<double> &p2,
                  std::vector<double> *p3, std::vector<Fep::QTor> &out) {
    auto &tt = lines(types);
    int maxe = 0;
    for (auto &l : tt) { auto v = line_values(l); long a; if (!v.empty() && to_int(v[0], a)) maxe = std::max<int>(maxe, (int)a); }
    fk.assign(maxe, 0); p2.assign(maxe, 0);
    if (p3) p3->assign(maxe, 0);
    for (auto &l : tt) {
      auto v = line_values(l);
      long j; double a, b, c = 0;
      size_t need = p3 ? 4 : 3;
      if (v.size() < need || !to_int(v[0], j) || j < 1 || !to_real(v[1], a) || !to_real(v[2], b) ||
          (p3 && !to_real(v[3], c)))
        bad(std::string(types) + ": " + l);
      fk[j - 1] = a;
      if (p3) { p2[j - 1] = b; (*p3)[j - 1] = deg2rad * c; }
      else p2[j - 1] = deg2rad * b;
    }
    for (auto &l : lines(changes)) {
      auto v = line_values(l);
      long a, b, c, d;
      if (v.size() < (size_t)(4 + S) || !to_int(v[0], a) || !to_int(v[1], b) || !to_int(v[2], c) || !to_int(v[3], d))
        bad(std::string(changes) + ": " + l);
      Fep::QTor q{(int)(a + f.offset) - 1, (int)(b + f.offset) - 1, (int)(c + f.offset) - 1, (int)(d + f.offset) - 1, {}};
      for (int s = 0; s < S; s++) {
        long cc;
        if (!to_int(v[4 + s], cc) || cc > maxe) bad(std::string(changes) + ": " + l);
        q.cod[s] = (int)cc;
      }
      out.push_back(q);
    }
  };
  tors("torsion_types", "change_torsions", f.qfktor, f.qrmult, &f.qdeltor, f.qtor);
  tors("improper_types", "change_impropers", f.qfkimp, f.qimp0, nullptr, f.qimp);
  // EVB couplings of Q angles, torsions and impropers to Morse Q bonds
  // (qatom.f90:1404-1497): "term bond", impropers "term bond [flag]"; the
  // bond must be Morse (no harmonic force constant) in every state it is in
  auto couplings = [&](const char *sec, size_t nterm, bool with_flag, std::vector<Fep::Coupling> &out) {
    for (auto &l : lines(sec)) {
      auto v = line_values(l);
      long j, k, fl = 0;
      if (v.size() < 2 || !to_int(v[0], j) || !to_int(v[1], k)) bad(std::string(sec) + ": " + l);
      if (with_flag && v.size() >= 3 && !to_int(v[2], fl)) fl = 0;
      if (j < 1 || j > (long)nterm || k < 1 || k > (long)f.qbnd.size()) bad(std::string(sec) + ": " + l);
      for (int s = 0; s < S; s++) {
        int c = f.qbnd[k - 1].cod[s];
        if (c > 0 && f.qbondlib[c - 1].fk != 0.0)
          bad(std::string(sec) + ": Q bond " + std::to_string(k) + " is harmonic in state " + std::to_string(s + 1));
      }
      out.push_back({(int)j - 1, (int)k - 1, (int)fl});
    }
  };
  couplings("angle_couplings", f.qang.size(), false, f.ang_coupl);
  couplings("torsion_couplings", f.qtor.size(), false, f.tor_coupl);
  couplings("improper_couplings", f.qimp.size(), true, f.imp_coupl);
  f.nang_coupl = (int)f.ang_coupl.size();
  f.ntor_coupl = (int)f.tor_coupl.size();
  f.nimp_coupl = (int)f.imp_coupl.size();
  for (auto &l : lines("shake_constraints")) {
    auto v = line_values(l);
    long a, b;
    if (v.size() < (size_t)(2 + S) || !to_int(v[0], a) || !to_int(v[1], b)) bad("shake_constraints: " + l);
    Fep::QShake q{(int)(a + f.offset) - 1, (int)(b + f.offset) - 1, {}};
    for (int s = 0; s < S; s++) if (!to_real(v[2 + s], q.dist[s])) bad("shake_constraints: " + l);
    f.qshake.push_back(q);
  }
  f.nqshake = (int)f.qshake.size();
  // off-diagonal functions "state_i state_j qatom_k qatom_l A_ij mu_ij" (qatom.f90:1515-1555)
  f.noffd = prm.count("off_diagonals");
  if (f.noffd > QB_MAX_STATES) fail(QB_ERR_PARSE, "too many off-diagonal functions (at most max_states)");
  for (auto &l : lines("off_diagonals")) {
    auto v = line_values(l);
    long i, j, k, q;
    double A, mu;
    if (v.size() < 6 || !to_int(v[0], i) || !to_int(v[1], j) || !to_int(v[2], k) || !to_int(v[3], q) ||
        !to_real(v[4], A) || !to_real(v[5], mu))
      bad("off_diagonals: " + l);
    if (i < 1 || i > S || j < 1 || j > S || i == j) bad("invalid combination of states in off_diagonals: " + l);
    if (k < 1 || k > f.nqat || q < 1 || q > f.nqat || f.iqseq[k - 1] < 0 || f.iqseq[q - 1] < 0)
      bad("invalid Q atoms in off_diagonals: " + l);
    f.offd.push_back({(int)i, (int)j, (int)k - 1, (int)q - 1, A, mu});
  }
  if (prm.count("monitor_groups") > 0 || prm.count("monitor_group_pairs") > 0)
    fail(QB_ERR_UNSUPPORTED, "monitor groups are not supported");
  // soft-core table (qatom.f90:1556-1685)
  const int ncol = t.natyps + nq;
  f.sc_lookup.assign((size_t)nq * ncol * S, 0.0);
  f.alpha_max.assign((size_t)nq * S, 0.0);
  if (auto sc = prm.section("softcore")) {
    if (!f.qvdw_flag) bad("softcore requires change_atoms");
    if ((int)sc->lines.size() != nq) bad("softcore must list every Q-atom");
    for (auto &l : sc->lines) {
      auto v = line_values(l);
      long iq;
      if (v.size() < (size_t)(1 + S) || !to_int(v[0], iq) || iq < 1 || iq > nq) bad("softcore: " + l);
      for (int s = 0; s < S; s++) if (!to_real(v[1 + s], f.alpha_max[(iq - 1) * S + s])) bad("softcore: " + l);
    }
    auto SC = [&](int iq, int col, int s) -> double & { return f.sc_lookup[((size_t)iq * ncol + col) * S + s]; };
    for (int i = 0; i < nq; i++) {
      for (int s = 0; s < S; s++) {
        double am = f.alpha_max[i * S + s];
        for (int j = 0; j < t.natyps; j++) {
          if (f.softcore_use_max_potential) {
            double aq = f.qavdw[f.qiac[i * S + s] * 3 + 0], bq = f.qbvdw[f.qiac[i * S + s] * 3 + 0];
            double aj = t.iaclib[j].avdw[0], bj = t.iaclib[j].bvdw[0];
            if (am != 0) {
              if (t.ivdw_rule == 2) {
                // arithmetic rule: bq is still epsilon, bj already sqrt(epsilon) (qatom.f90:1618-1622)
                double s6 = (aq + aj) * (aq + aj);
                s6 = s6 * s6 * s6;
                SC(i, j, s) = (-2 * std::sqrt(bq) * bj + 2 * std::sqrt(bq * bj * bj + am * std::sqrt(bq) * bj)) *
                              s6 / (2 * am);
              } else {
                SC(i, j, s) = (-bq * bj + std::sqrt(bq * bq * bj * bj + 4 * am * aq * aj)) / (2 * am);
              }
            }
          } else {
            SC(i, j, s) = am;
          }
        }
        for (int j = 0; j < nq; j++) {
          double amj = f.alpha_max[j * S + s];
          if (am > 1e-6 || amj > 1e-6) {
            double aq = f.qavdw[f.qiac[i * S + s] * 3 + 0], bq = f.qbvdw[f.qiac[i * S + s] * 3 + 0];
            double aj = f.qavdw[f.qiac[j * S + s] * 3 + 0], bj = f.qbvdw[f.qiac[j * S + s] * 3 + 0];
            double tmp;
            if (f.softcore_use_max_potential) {
              tmp = std::min(am, amj);
              if (am == 0 || amj == 0) tmp = std::max(am, amj);
              if (t.ivdw_rule == 2) {
                // arithmetic rule: both epsilons not yet square-rooted (qatom.f90:1660-1664)
                double s6 = (aq + aj) * (aq + aj);
                s6 = s6 * s6 * s6;
                SC(i, j + t.natyps, s) =
                    (-2 * std::sqrt(bq * bj) + 2 * std::sqrt(bq * bj + tmp * std::sqrt(bq * bj))) * s6 / (2 * tmp);
              } else {
                SC(i, j + t.natyps, s) = (-bq * bj + std::sqrt(bq * bq * bj * bj + 4 * tmp * aq * aj)) / (2 * tmp);
              }
            } else {
              SC(i, j + t.natyps, s) = std::max(am, amj);
            }
          }
        }
      }
    }
  }
}

// ------------------------------------------------------------ restart file

namespace {
void write_record(std::FILE *f, const void *const *parts, const size_t *sizes, int n) {
  uint32_t len = 0;
  for (int i = 0; i < n; i++) len += (uint32_t)sizes[i];
  std::fwrite(&len, 4, 1, f);
  for (int i = 0; i < n; i++) std::fwrite(parts[i], 1, sizes[i], f);
  std::fwrite(&len, 4, 1, f);
}

bool read_record(std::FILE *f, std::vector<char> &buf) {
  uint32_t len, len2;
  if (std::fread(&len, 4, 1, f) != 1) return false;
  buf.resize(len);
  if (len && std::fread(buf.data(), 1, len, f) != len) return false;
  if (std::fread(&len2, 4, 1, f) != 1 || len2 != len) return false;
  return true;
}
}  // namespace

void read_restart(const std::string &path, int natom, std::vector<double> &x, std::vector<double> &v,
                  int nshell, std::vector<float> *theta_corr, double *boxl, double *boxc) {
  std::FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) fail(QB_ERR_IO, "cannot open restart file " + path);
  std::vector<char> rec;
  auto vec = [&](std::vector<double> &out, const char *what) {
    if (!read_record(f, rec) || rec.size() < 4) { std::fclose(f); fail(QB_ERR_PARSE, path + ": truncated restart (" + what + ")"); }
    int32_t nat3;
    std::memcpy(&nat3, rec.data(), 4);
    if (nat3 != 3 * natom) { std::fclose(f); fail(QB_ERR_PARSE, path + ": wrong number of atoms in restart file"); }
    if (rec.size() != 4 + 8 * (size_t)nat3) { std::fclose(f); fail(QB_ERR_PARSE, path + ": bad record length"); }
    out.resize(nat3);
    std::memcpy(out.data(), rec.data() + 4, 8 * (size_t)nat3);
  };
  vec(x, "coordinates");
  vec(v, "velocities");
  if (boxl) {
    // periodic box: (boxlength), (boxcenter) follow the velocities
    double *dst[2] = {boxl, boxc};
    for (int r = 0; r < 2; r++) {
      if (!read_record(f, rec) || rec.size() != 24) { std::fclose(f); fail(QB_ERR_PARSE, path + ": restart file lacks the box records"); }
      std::memcpy(dst[r], rec.data(), 24);
    }
  }
  if (theta_corr && nshell > 0) {
    // wat_shells (md.f90:15068-15082): use the record only if its shell count matches
    if (read_record(f, rec) && rec.size() == 4 + 4 * (size_t)nshell) {
      int32_t ns;
      std::memcpy(&ns, rec.data(), 4);
      if (ns == nshell) {
        theta_corr->resize(nshell);
        std::memcpy(theta_corr->data(), rec.data() + 4, 4 * (size_t)nshell);
      }
    }
  }
  std::fclose(f);
}

void write_restart(const std::string &path, int natom, const double *x, const double *v, int nshell,
                   const float *theta_corr, const double *box6) {
  std::FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) fail(QB_ERR_IO, "cannot write " + path);
  int32_t nat3 = 3 * natom;
  {
    const void *p[2] = {&nat3, x};
    size_t s[2] = {4, 8 * (size_t)nat3};
    write_record(f, p, s, 2);
  }
  {
    const void *p[2] = {&nat3, v};
    size_t s[2] = {4, 8 * (size_t)nat3};
    write_record(f, p, s, 2);
  }
  if (nshell > 0 && theta_corr) {
    int32_t ns = nshell;
    const void *p[2] = {&ns, theta_corr};
    size_t s[2] = {4, 4 * (size_t)nshell};
    write_record(f, p, s, 2);
  }
  if (box6) {
    // write_xfin's box records (md.f90:15471-15474): edge lengths, centre
    for (int r = 0; r < 2; r++) {
      const void *p[1] = {box6 + 3 * r};
      size_t s[1] = {24};
      write_record(f, p, s, 1);
    }
  }
  std::fclose(f);
}

void append_energy_frame(const std::string &path, int nstates, const double *EQ, int noffd, const int *ij,
                         const double *hr) {
  std::FILE *f = std::fopen(path.c_str(), "ab");
  if (!f) fail(QB_ERR_IO, "cannot write " + path);
  for (int s = 0; s < nstates; s++) {
    int32_t i = s + 1;
    const void *p[2] = {&i, EQ + (size_t)s * QB_NEQ};
    size_t sz[2] = {4, 8 * (size_t)QB_NEQ};
    write_record(f, p, sz, 2);
  }
  // off-diagonal record: noffd x (int32 i, int32 j, real8 Hij, real8 rkl), nrgy.f90:60-65, 116
  std::vector<char> od((size_t)noffd * 24);
  for (int k = 0; k < noffd; k++) {
    int32_t ij32[2] = {ij[2 * k], ij[2 * k + 1]};
    std::memcpy(od.data() + 24 * k, ij32, 8);
    std::memcpy(od.data() + 24 * k + 8, hr + 2 * k, 16);
  }
  const void *p[1] = {od.data()};
  size_t sz[1] = {od.size()};
  write_record(f, p, sz, noffd > 0 ? 1 : 0);
  std::fclose(f);
}

}  // namespace qb
