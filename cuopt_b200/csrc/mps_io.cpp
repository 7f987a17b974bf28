// MPS input/output for cuOptReadProblem / cuOptWriteProblem.
//
// Conventions follow the reference parser (cpp/libmps_parser/src/mps_parser.cpp):
//   * the first N row is the objective, its RHS entry is the negated objective offset (:1098);
//   * RANGES: E row with R < 0 -> [b + R, b], R >= 0 -> [b, b + R]; G row -> [b, b + |R|];
//     L row -> [b - |R|, b] (:354-405);
//   * BOUNDS LO/UP/FX/FR/MI/PL/BV/LI/UI; an UP bound below 0 on a variable without an earlier
//     bound sets the lower bound to -inf (:1386-1393);
//   * default variable bounds [0, +inf); MARKER INTORG/INTEND marks integer columns.
// Records follow the reference's free-format rules (cuOptReadProblem parses free MPS,
// cpp/src/pdlp/cuopt_c.cpp:103-107), which fixed-format files without blanks in names also meet:
//   * a line starting with '*' or '$' is a comment; in a data line a field starting with '$'
//     ends the record (:594-597, 974-978, 1077-1082, 1133-1154, 1196);
//   * a line starting with anything but a blank opens a section (:599);
//   * OBJNAME (on its line or the next) names the objective and must come before ROWS
//     (:1262-1281); further N rows are ignored, with their COLUMNS entries (:840-859, 1005);
//   * duplicate rows and columns whose entries are not contiguous are errors (:863, 913);
//   * RHS records name a set unless the first field is a row or the objective (:1050-1060);
//     RANGES records always name a set (:1192-1193); a BOUNDS record leaves the set name out
//     when its second field is a column, and may define a column (:1136-1167);
//   * OBJSENSE takes MIN / MINIMIZE / MAX / MAXIMIZE only (:257-270);
//   * an objective row and the ROWS, COLUMNS and RHS sections are required (:772-780);
//   * integer columns without any bound get [0, 1] (:801-806).
// Compressed files are not supported.
#include <cuopt/linear_programming/constants.h>

#include <cmath>
#include <cstdio>
#include <fstream>
#include <limits>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "lp_model.hpp"

namespace cuopt_b200 {

namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();

// Whitespace-separated fields up to the first one that starts with '$' (the rest of the line is a
// comment); `cut` tells whether such a field was met.
std::vector<std::string> split(const std::string& line, bool& cut)
{
  std::vector<std::string> t;
  std::istringstream ss(line);
  std::string w;
  cut = false;
  while (ss >> w) {
    if (w[0] == '$') {
      cut = true;
      break;
    }
    t.push_back(w);
  }
  return t;
}

bool to_double(const std::string& s, double& v)
{
  try {
    size_t pos = 0;
    v          = std::stod(s, &pos);
    return pos == s.size();
  } catch (const std::exception&) {
    return false;
  }
}

}  // namespace

int read_mps(const std::string& path, lp_problem& out, std::string& err)
{
  std::ifstream f(path);
  if (!f.is_open()) {
    err = "Error opening MPS file";
    return CUOPT_MPS_FILE_ERROR;
  }
  enum sec { NONE, NAME, OBJSENSE, OBJNAME, ROWS, COLUMNS, RHS, RANGES, BOUNDS, END } cur = NONE;
  std::string obj_row;
  std::set<std::string> ignored_obj;  // N rows after the objective
  bool seen_rows = false, seen_columns = false, seen_rhs = false;
  std::vector<std::string> row_names;
  std::vector<char> row_types;
  std::unordered_map<std::string, int> row_id, col_id;
  std::vector<std::string> col_names;
  std::vector<std::vector<std::pair<int, double>>> cols;  // entries per column
  std::vector<double> cost, rhs, ranges, lo, up;
  std::vector<char> vtype;
  std::set<int> bounded;
  bool integer_block = false, maximize = false;
  double offset      = 0.0;
  const double unset = std::numeric_limits<double>::quiet_NaN();
  std::string line;
  int lineno = 0;
  auto fail = [&](const std::string& what) {
    err = what + " (line " + std::to_string(lineno) + ")";
    return CUOPT_MPS_PARSE_ERROR;
  };
  auto col_of = [&](const std::string& name) {
    auto it = col_id.find(name);
    if (it != col_id.end()) return it->second;
    const int id = (int)col_names.size();
    col_id.emplace(name, id);
    col_names.push_back(name);
    cols.emplace_back();
    cost.push_back(0.0);
    lo.push_back(0.0);
    up.push_back(kInf);
    vtype.push_back(integer_block ? 'I' : 'C');
    return id;
  };
  auto set_sense = [&](const std::string& w) {
    if (w == "MIN" || w == "MINIMIZE") maximize = false;
    else if (w == "MAX" || w == "MAXIMIZE") maximize = true;
    else return false;
    return true;
  };
  auto set_objname = [&](const std::string& w) {
    if (!obj_row.empty()) return false;  // OBJNAME must precede ROWS
    obj_row = w;
    return true;
  };
  while (std::getline(f, line)) {
    ++lineno;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.empty() || line[0] == '*' || line[0] == '$') continue;
    bool cut  = false;
    auto tok  = split(line, cut);
    if (tok.empty()) continue;
    if (line[0] != ' ') {
      const std::string& h = tok[0];
      if (h == "NAME") {
        cur = NAME;
        if (tok.size() > 1) out.name = tok[1];
        continue;
      }
      if (h == "OBJSENSE") {
        cur = OBJSENSE;
        if (tok.size() > 1 && !set_sense(tok[1])) return fail("Bad OBJSENSE " + tok[1]);
        continue;
      }
      if (h == "OBJNAME") {
        cur = OBJNAME;
        if (tok.size() > 1 && !set_objname(tok[1]))
          return fail("OBJNAME must come before the ROWS section");
        continue;
      }
      if (h == "ROWS") { cur = ROWS; seen_rows = true; continue; }
      if (h == "COLUMNS") { cur = COLUMNS; seen_columns = true; continue; }
      if (h == "RHS") {
        cur      = RHS;
        seen_rhs = true;
        if (rhs.empty()) rhs.assign(row_names.size(), 0.0);
        continue;
      }
      if (h == "RANGES") {
        cur = RANGES;
        ranges.assign(row_names.size(), unset);
        continue;
      }
      if (h == "BOUNDS") { cur = BOUNDS; continue; }
      if (h == "ENDATA") { cur = END; break; }
      return fail("Unknown section " + h);
    }
    switch (cur) {
      case OBJSENSE:
        if (!set_sense(tok[0])) return fail("Bad OBJSENSE " + tok[0]);
        break;
      case OBJNAME:
        if (!set_objname(tok[0])) return fail("OBJNAME must come before the ROWS section");
        break;
      case ROWS: {
        if (tok.size() < 2) return fail("Bad ROWS line");
        const std::string& t = tok[0];
        if (t == "N") {
          if (obj_row.empty()) obj_row = tok[1];
          else if (tok[1] != obj_row) ignored_obj.insert(tok[1]);
          break;
        }
        if (t != "E" && t != "L" && t != "G") return fail("Bad row type " + t);
        if (!row_id.emplace(tok[1], (int)row_names.size()).second)
          return fail("Duplicate row " + tok[1]);
        row_names.push_back(tok[1]);
        row_types.push_back(t[0]);
        break;
      }
      case COLUMNS: {
        if (tok.size() >= 3 && (tok[1] == "'MARKER'" || tok[1] == "MARKER")) {
          if (tok[2] == "'INTORG'") integer_block = true;
          if (tok[2] == "'INTEND'") integer_block = false;
          break;
        }
        // A record cut short by a comment after the column name only names the column.
        if (tok.size() % 2 == 0) return fail("Bad COLUMNS line");
        auto known = col_id.find(tok[0]);
        if (known != col_id.end() && known->second != (int)col_names.size() - 1)
          return fail("Entries of column " + tok[0] + " are not contiguous");
        const int j = col_of(tok[0]);
        for (size_t q = 1; q + 1 < tok.size(); q += 2) {
          double v;
          if (!to_double(tok[q + 1], v)) return fail("Bad value in COLUMNS");
          if (tok[q] == obj_row) {
            cost[j] = v;
            continue;
          }
          if (ignored_obj.count(tok[q])) continue;
          auto it = row_id.find(tok[q]);
          if (it == row_id.end()) return fail("Unknown row " + tok[q]);
          cols[j].emplace_back(it->second, v);
        }
        break;
      }
      case RHS:
      case RANGES: {
        size_t q;
        if (cur == RHS) q = (tok[0] == obj_row || row_id.count(tok[0])) ? 0 : 1;
        else q = 1;
        if ((tok.size() - q) % 2 != 0) return fail("Bad RHS/RANGES line");  // tok.size() >= 1 >= q
        for (; q + 1 < tok.size(); q += 2) {
          double v;
          if (!to_double(tok[q + 1], v)) return fail("Bad value in RHS/RANGES");
          if (cur == RHS && tok[q] == obj_row) {
            offset = -v;
            continue;
          }
          auto it = row_id.find(tok[q]);
          if (it == row_id.end()) return fail("Unknown row " + tok[q]);
          (cur == RHS ? rhs : ranges)[it->second] = v;
        }
        break;
      }
      case BOUNDS: {
        const std::string& t = tok[0];
        const bool novalue   = (t == "FR" || t == "MI" || t == "PL" || t == "BV");
        // The bound set name is left out when the second field is a column.
        const size_t vi = (tok.size() > 1 && col_id.count(tok[1])) ? 1 : 2;
        if (tok.size() <= vi) {
          if (cut) break;  // the column field is a comment
          return fail("Bad BOUNDS line");
        }
        const std::string cname = tok[vi];
        double v                = 0.0;
        if (!novalue) {
          if (tok.size() <= vi + 1) return fail("Bad BOUNDS line");
          if (!to_double(tok[vi + 1], v)) return fail("Bad value in BOUNDS");
        }
        const int j = col_of(cname);  // a column named only here has no entries
        if (t == "LO") lo[j] = v;
        else if (t == "UP" || t == "UI") {
          up[j] = v;
          if (!bounded.count(j) && v < 0) lo[j] = -kInf;
          if (t == "UI") vtype[j] = 'I';
        } else if (t == "FX") {
          lo[j] = v;
          up[j] = v;
        } else if (t == "FR") {
          lo[j] = -kInf;
          up[j] = kInf;
        } else if (t == "MI") lo[j] = -kInf;
        else if (t == "PL") up[j] = kInf;
        else if (t == "BV") {
          lo[j]    = 0;
          up[j]    = 1;
          vtype[j] = 'I';
        } else if (t == "LI") {
          if (!bounded.count(j)) up[j] = kInf;
          lo[j]    = v;
          vtype[j] = 'I';
        } else
          return fail("Unsupported bound type " + t);
        bounded.insert(j);
        break;
      }
      default: return fail("Data outside a section");
    }
  }
  if (obj_row.empty()) return fail("No objective row");
  if (!seen_rows) return fail("ROWS section missing");
  if (!seen_columns) return fail("COLUMNS section missing");
  if (!seen_rhs) return fail("RHS section missing");
  // Integer columns without any bound are binary (reference mps_parser.cpp:801-806).
  for (int j = 0; j < (int)col_names.size(); ++j)
    if (vtype[j] == 'I' && !bounded.count(j)) {
      lo[j] = 0.0;
      up[j] = 1.0;
    }
  const int m = (int)row_names.size(), n = (int)col_names.size();
  if (rhs.empty()) rhs.assign(m, 0.0);
  out.m          = m;
  out.n          = n;
  out.maximize   = maximize;
  out.obj_offset = offset;
  out.c.assign(cost.begin(), cost.end());
  out.var_lo.assign(lo.begin(), lo.end());
  out.var_up.assign(up.begin(), up.end());
  out.var_types  = vtype;
  out.row_names  = row_names;
  out.col_names  = col_names;
  out.objective_name = obj_row;
  out.row_types  = row_types;
  out.rhs.assign(rhs.begin(), rhs.end());
  out.ranged     = true;
  out.con_lo.resize(m);
  out.con_up.resize(m);
  for (int i = 0; i < m; ++i) {
    const double b = rhs[i];
    double l = -kInf, u = kInf;
    if (row_types[i] == 'E') l = u = b;
    if (row_types[i] == 'G') l = b;
    if (row_types[i] == 'L') u = b;
    if (!ranges.empty() && !std::isnan(ranges[i])) {
      const double r = ranges[i];
      if (row_types[i] == 'E') {
        if (r < 0) l = b + r;
        else u = b + r;
      } else if (row_types[i] == 'G') {
        u = l + std::fabs(r);
      } else {
        l = u - std::fabs(r);
      }
    }
    out.con_lo[i] = l;
    out.con_up[i] = u;
  }
  // CSR from the column lists.
  out.row_off.assign(m + 1, 0);
  for (int j = 0; j < n; ++j)
    for (auto& e : cols[j]) out.row_off[e.first + 1]++;
  for (int i = 0; i < m; ++i) out.row_off[i + 1] += out.row_off[i];
  out.col_idx.resize(out.row_off[m]);
  out.val.resize(out.row_off[m]);
  std::vector<int> fillp(out.row_off.begin(), out.row_off.end() - 1);
  for (int j = 0; j < n; ++j)
    for (auto& e : cols[j]) {
      const int d     = fillp[e.first]++;
      out.col_idx[d] = j;
      out.val[d]     = e.second;
    }
  return CUOPT_SUCCESS;
}

int write_sol_file(const lp_problem& p, lp_solution& s, const std::string& path)
{
  std::ofstream f(path);
  if (!f.is_open()) return CUOPT_INVALID_ARGUMENT;
  const int st        = s.r.status;
  const bool feasible = st == CUOPT_TERIMINATION_STATUS_OPTIMAL ||
                        st == CUOPT_TERIMINATION_STATUS_PRIMAL_FEASIBLE;
  f.precision(std::numeric_limits<double>::max_digits10 + 1);
  f << "# Status: "
    << (st == CUOPT_TERIMINATION_STATUS_OPTIMAL ? "Optimal"
                                                : (feasible ? "Primal Feasible" : "Infeasible"))
    << "\n";
  if (!feasible) return CUOPT_SUCCESS;
  f << "# Objective value: " << s.r.primal_obj << "\n";
  ensure_host(s.r);
  for (size_t j = 0; j < p.col_names.size() && j < s.r.x.size(); ++j)
    f << p.col_names[j] << " " << s.r.x[j] << "\n";
  return f.good() ? CUOPT_SUCCESS : CUOPT_INVALID_ARGUMENT;
}

int write_mps(const lp_problem& p, const std::string& path)
{
  std::FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return CUOPT_MPS_FILE_ERROR;
  std::vector<double> lo, up;
  p.constraint_bounds(lo, up);
  auto rname = [&](int i) {
    return i < (int)p.row_names.size() ? p.row_names[i] : "R" + std::to_string(i);
  };
  auto cname = [&](int j) {
    return j < (int)p.col_names.size() ? p.col_names[j] : "C" + std::to_string(j);
  };
  std::fprintf(f, "NAME %s\n", p.name.empty() ? "PROBLEM" : p.name.c_str());
  if (p.maximize) std::fprintf(f, "OBJSENSE\n    MAX\n");
  std::fprintf(f, "ROWS\n N  OBJ\n");
  std::vector<char> t(p.m);
  for (int i = 0; i < p.m; ++i) {
    if (lo[i] == up[i]) t[i] = 'E';
    else if (std::isinf(lo[i])) t[i] = 'L';
    else t[i] = 'G';
    std::fprintf(f, " %c  %s\n", t[i], rname(i).c_str());
  }
  std::vector<std::vector<std::pair<int, double>>> cols(p.n);
  for (int i = 0; i < p.m; ++i)
    for (int k = p.row_off[i]; k < p.row_off[i + 1]; ++k) cols[p.col_idx[k]].emplace_back(i, p.val[k]);
  std::fprintf(f, "COLUMNS\n");
  bool in_int = false;
  for (int j = 0; j < p.n; ++j) {
    const bool is_int = j < (int)p.var_types.size() && p.var_types[j] == 'I';
    if (is_int != in_int) {
      std::fprintf(f, "    MARKER  'MARKER'  '%s'\n", is_int ? "INTORG" : "INTEND");
      in_int = is_int;
    }
    std::fprintf(f, "    %s  OBJ  %.17g\n", cname(j).c_str(), p.c[j]);
    for (auto& e : cols[j]) std::fprintf(f, "    %s  %s  %.17g\n", cname(j).c_str(), rname(e.first).c_str(), e.second);
  }
  if (in_int) std::fprintf(f, "    MARKER  'MARKER'  'INTEND'\n");
  std::fprintf(f, "RHS\n");
  if (p.obj_offset != 0.0) std::fprintf(f, "    RHS  OBJ  %.17g\n", -p.obj_offset);
  for (int i = 0; i < p.m; ++i) {
    const double b = (t[i] == 'L') ? up[i] : lo[i];
    if (b != 0.0) std::fprintf(f, "    RHS  %s  %.17g\n", rname(i).c_str(), b);
  }
  bool any_range = false;
  for (int i = 0; i < p.m; ++i)
    if (t[i] == 'G' && std::isfinite(up[i])) any_range = true;
  if (any_range) {
    std::fprintf(f, "RANGES\n");
    for (int i = 0; i < p.m; ++i)
      if (t[i] == 'G' && std::isfinite(up[i]))
        std::fprintf(f, "    RNG  %s  %.17g\n", rname(i).c_str(), up[i] - lo[i]);
  }
  std::fprintf(f, "BOUNDS\n");
  for (int j = 0; j < p.n; ++j) {
    const double l = p.var_lo[j], u = p.var_up[j];
    const std::string c = cname(j);
    if (l == u) {
      std::fprintf(f, " FX BND  %s  %.17g\n", c.c_str(), l);
      continue;
    }
    if (std::isinf(l) && std::isinf(u)) {
      std::fprintf(f, " FR BND  %s\n", c.c_str());
      continue;
    }
    if (std::isinf(l)) std::fprintf(f, " MI BND  %s\n", c.c_str());
    else if (l != 0.0) std::fprintf(f, " LO BND  %s  %.17g\n", c.c_str(), l);
    if (std::isfinite(u)) std::fprintf(f, " UP BND  %s  %.17g\n", c.c_str(), u);
  }
  std::fprintf(f, "ENDATA\n");
  std::fclose(f);
  return CUOPT_SUCCESS;
}

}  // namespace cuopt_b200
