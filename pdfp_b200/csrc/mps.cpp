// mps.cpp -- MPS files (plain or gzip) into the pump's canonical MILP.
//
// The reference reads MPS through QPSReader and canonicalises in
// src/milp.jl:42-94: a maximisation objective is negated; binaries get bounds
// clipped to [0, 1]; a row with equal finite bounds becomes an equality row;
// otherwise a finite upper bound gives A_i x <= hi and a finite lower bound
// gives -A_i x <= -lo, in that order; |values| >= 1e20 are infinite.  This is
// the same reading as pdfp_b200/milp.py:read_mps (free MPS: whitespace-separated
// fields; default bounds [0, inf); integer columns from MARKER INTORG/INTEND
// blocks and LI/UI/BV bounds; the objective constant is minus the objective
// row's RHS), in C++ so that large instances -- the SCIP-presolved MIPLIB files
// of benchmark/presolve are MPS too -- load without the interpreter.
#include <zlib.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/pdfp_b200.h"
#include "device.hpp"
#include "mps.hpp"

namespace pdfp {

namespace {

constexpr double kMpsInfinity = 1.0e20;  // src/milp.jl:36
const double kInf = std::numeric_limits<double>::infinity();

bool is_infinite(double v) { return !std::isfinite(v) || std::fabs(v) >= kMpsInfinity; }

std::string upper(std::string s) {
    for (char& ch : s) ch = static_cast<char>(std::toupper(static_cast<unsigned char>(ch)));
    return s;
}

std::string strip_quotes(const std::string& s) {
    size_t a = 0, e = s.size();
    while (a < e && (s[a] == '\'' || s[a] == '"')) ++a;
    while (e > a && (s[e - 1] == '\'' || s[e - 1] == '"')) --e;
    return s.substr(a, e - a);
}

double to_double(const std::string& s, int line) {
    char* end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (end == s.c_str() || *end != '\0')
        throw Error(E_INVALID, "MPS line " + std::to_string(line) + ": bad number '" + s + "'");
    return v;
}

void split(const char* line, std::vector<std::string>& tok) {
    tok.clear();
    const char* p = line;
    while (*p) {
        while (*p && std::isspace(static_cast<unsigned char>(*p))) ++p;
        if (!*p) break;
        const char* q = p;
        while (*q && !std::isspace(static_cast<unsigned char>(*q))) ++q;
        tok.emplace_back(p, q);
        p = q;
    }
}

struct GzFile {
    gzFile f = nullptr;
    ~GzFile() {
        if (f) gzclose(f);
    }
};

}  // namespace

MpsModel* read_mps_file(const char* path) {
    GzFile fh;
    fh.f = gzopen(path, "rb");
    if (!fh.f) throw Error(E_INVALID, std::string("cannot open ") + path);
    gzbuffer(fh.f, 1 << 20);

    std::vector<char> rtype;  // per constraint row, file order (objective excluded)
    std::unordered_map<std::string, int32_t> row_index, col_index;
    std::string obj_row;
    bool have_obj = false;
    std::vector<uint8_t> col_int;
    std::vector<int32_t> tr, tc;
    std::vector<double> tv;
    std::unordered_map<int32_t, double> c_vals, rhs, ranges, lvar, uvar;
    std::unordered_set<int32_t> binary, explicit_int;
    double c0 = 0.0;
    bool maximise = false, in_int = false;
    std::string section;

    auto col_id = [&](const std::string& name) -> int32_t {
        auto it = col_index.find(name);
        if (it != col_index.end()) return it->second;
        const int32_t j = static_cast<int32_t>(col_int.size());
        col_index.emplace(name, j);
        col_int.push_back(in_int ? 1 : 0);
        return j;
    };

    std::string line;
    std::vector<std::string> tok;
    std::vector<char> buf(1 << 16);
    int lineno = 0;
    bool done = false;
    while (!done) {
        // one logical line, however long
        line.clear();
        bool got = false;
        while (gzgets(fh.f, buf.data(), static_cast<int>(buf.size())) != nullptr) {
            got = true;
            line.append(buf.data());
            if (!line.empty() && line.back() == '\n') break;
        }
        if (!got) break;
        ++lineno;
        while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
        size_t first = line.find_first_not_of(" \t");
        if (first == std::string::npos || line[first] == '*') continue;
        split(line.c_str(), tok);
        if (!std::isspace(static_cast<unsigned char>(line[0]))) {
            section = upper(tok[0]);
            if (section == "OBJSENSE" && tok.size() > 1) maximise = upper(tok[1]).rfind("MAX", 0) == 0;
            if (section == "ENDATA") done = true;
            continue;
        }
        if (section == "OBJSENSE") {
            maximise = upper(tok[0]).rfind("MAX", 0) == 0;
        } else if (section == "ROWS") {
            if (tok.size() < 2) throw Error(E_INVALID, "MPS line " + std::to_string(lineno) + ": short ROWS entry");
            const std::string t = upper(tok[0]);
            if (t == "N") {
                if (!have_obj) {
                    obj_row = tok[1];
                    have_obj = true;
                }
                continue;  // further free rows carry no constraint
            }
            if (t != "L" && t != "G" && t != "E")
                throw Error(E_INVALID, "MPS line " + std::to_string(lineno) + ": unknown row type " + t);
            row_index.emplace(tok[1], static_cast<int32_t>(rtype.size()));
            rtype.push_back(t[0]);
        } else if (section == "COLUMNS") {
            if (tok.size() >= 3 && upper(strip_quotes(tok[1])) == "MARKER") {
                const std::string mk = upper(strip_quotes(tok[2]));
                if (mk == "INTORG") in_int = true;
                else if (mk == "INTEND") in_int = false;
                continue;
            }
            const int32_t j = col_id(tok[0]);
            for (size_t k = 1; k + 1 < tok.size(); k += 2) {
                const double val = to_double(tok[k + 1], lineno);
                if (have_obj && tok[k] == obj_row) {
                    c_vals[j] += val;
                } else {
                    auto it = row_index.find(tok[k]);
                    if (it != row_index.end()) {
                        tr.push_back(it->second);
                        tc.push_back(j);
                        tv.push_back(val);
                    }
                }
            }
        } else if (section == "RHS" || section == "RANGES") {
            const size_t k0 = tok.size() % 2 == 1 ? 1 : 0;  // optional set name
            for (size_t k = k0; k + 1 < tok.size(); k += 2) {
                const double val = to_double(tok[k + 1], lineno);
                if (section == "RHS") {
                    if (have_obj && tok[k] == obj_row) {
                        c0 = -val;
                    } else {
                        auto it = row_index.find(tok[k]);
                        if (it != row_index.end()) rhs[it->second] = val;
                    }
                } else {
                    auto it = row_index.find(tok[k]);
                    if (it != row_index.end()) ranges[it->second] = val;
                }
            }
        } else if (section == "BOUNDS") {
            const std::string bt = upper(tok[0]);
            const bool needs_value = bt == "UP" || bt == "LO" || bt == "FX" || bt == "LI" || bt == "UI" || bt == "SC";
            std::string cname;
            double val = 0.0;
            if (needs_value) {
                if (tok.size() >= 4) {
                    cname = tok[2];
                    val = to_double(tok[3], lineno);
                } else if (tok.size() == 3) {
                    cname = tok[1];
                    val = to_double(tok[2], lineno);
                } else {
                    throw Error(E_INVALID, "MPS line " + std::to_string(lineno) + ": short BOUNDS entry");
                }
            } else {
                if (tok.size() < 2) throw Error(E_INVALID, "MPS line " + std::to_string(lineno) + ": short BOUNDS entry");
                cname = tok.size() >= 3 ? tok[2] : tok[1];
            }
            const int32_t j = col_id(cname);
            if (bt == "UP") {
                uvar[j] = val;
                if (val < 0 && lvar.find(j) == lvar.end()) lvar[j] = -kInf;
            } else if (bt == "LO") {
                lvar[j] = val;
            } else if (bt == "FX") {
                lvar[j] = val;
                uvar[j] = val;
            } else if (bt == "FR") {
                lvar[j] = -kInf;
                uvar[j] = kInf;
            } else if (bt == "MI") {
                lvar[j] = -kInf;
            } else if (bt == "PL") {
                uvar[j] = kInf;
            } else if (bt == "BV") {
                binary.insert(j);
                lvar[j] = 0.0;
                uvar[j] = 1.0;
            } else if (bt == "LI") {
                explicit_int.insert(j);
                lvar[j] = val;
            } else if (bt == "UI") {
                explicit_int.insert(j);
                uvar[j] = val;
            } else if (bt == "SC") {
                uvar[j] = val;
            }
        }
    }

    std::unique_ptr<MpsModel> M(new MpsModel());
    const int32_t n = static_cast<int32_t>(col_int.size());
    const double sign = maximise ? -1.0 : 1.0;
    M->n = n;
    M->c.assign(n, 0.0);
    for (const auto& kv : c_vals) M->c[kv.first] = kv.second;
    for (double& x : M->c) x = sign * x;
    M->c0 = sign * c0;
    M->l.assign(n, 0.0);
    M->u.assign(n, kInf);
    for (const auto& kv : lvar) M->l[kv.first] = kv.second;
    for (const auto& kv : uvar) M->u[kv.first] = kv.second;
    for (int32_t j = 0; j < n; ++j) {
        if (is_infinite(M->l[j])) M->l[j] = M->l[j] < 0 ? -kInf : kInf;
        if (is_infinite(M->u[j])) M->u[j] = M->u[j] < 0 ? -kInf : kInf;
        if (binary.count(j)) {
            M->int_idx.push_back(j);
            M->l[j] = std::max(M->l[j], 0.0);
            M->u[j] = std::min(M->u[j], 1.0);
        } else if (col_int[j] || explicit_int.count(j)) {
            M->int_idx.push_back(j);
        }
    }

    // canonical rows of each original row (src/milp.jl:66-83): (row, sign)
    const int32_t R = static_cast<int32_t>(rtype.size());
    std::vector<int32_t> can_first(R, -1), can_count(R, 0);
    std::vector<double> can_sign;
    for (int32_t i = 0; i < R; ++i) {
        auto it = rhs.find(i);
        const double r = it == rhs.end() ? 0.0 : it->second;
        double lo, hi;
        auto rg = ranges.find(i);
        if (rtype[i] == 'E') {
            lo = hi = r;
            if (rg != ranges.end()) {
                const double Rv = rg->second;
                if (Rv > 0) hi = r + std::fabs(Rv);
                else lo = r - std::fabs(Rv);
            }
        } else if (rtype[i] == 'L') {
            lo = -kInf;
            hi = r;
            if (rg != ranges.end()) lo = r - std::fabs(rg->second);
        } else {
            lo = r;
            hi = kInf;
            if (rg != ranges.end()) hi = r + std::fabs(rg->second);
        }
        can_first[i] = static_cast<int32_t>(M->b.size());
        if (!is_infinite(lo) && !is_infinite(hi) && lo == hi) {
            M->b.push_back(hi);
            M->is_eq.push_back(1);
            can_sign.push_back(1.0);
            can_count[i] = 1;
            continue;
        }
        if (!is_infinite(hi)) {
            M->b.push_back(hi);
            M->is_eq.push_back(0);
            can_sign.push_back(1.0);
            ++can_count[i];
        }
        if (!is_infinite(lo)) {
            M->b.push_back(-lo);
            M->is_eq.push_back(0);
            can_sign.push_back(-1.0);
            ++can_count[i];
        }
    }
    M->m = static_cast<int32_t>(M->b.size());

    // CSR of the canonical rows: entries of each row by ascending column,
    // duplicates summed in file order
    std::vector<int64_t> cnt(static_cast<size_t>(M->m) + 1, 0);
    for (size_t t = 0; t < tr.size(); ++t)
        for (int32_t q = 0; q < can_count[tr[t]]; ++q) ++cnt[can_first[tr[t]] + q + 1];
    for (int32_t i = 0; i < M->m; ++i) cnt[i + 1] += cnt[i];
    if (cnt[M->m] > std::numeric_limits<int32_t>::max())
        throw Error(E_UNSUPPORTED, "more than 2^31 - 1 nonzeros");
    std::vector<int32_t> col(static_cast<size_t>(cnt[M->m]));
    std::vector<double> val(static_cast<size_t>(cnt[M->m]));
    std::vector<int64_t> next(cnt.begin(), cnt.end() - 1);
    for (size_t t = 0; t < tr.size(); ++t)
        for (int32_t q = 0; q < can_count[tr[t]]; ++q) {
            const int32_t row = can_first[tr[t]] + q;
            const int64_t p = next[row]++;
            col[p] = tc[t];
            val[p] = can_sign[row] * tv[t];
        }
    M->rp.assign(static_cast<size_t>(M->m) + 1, 0);
    std::vector<std::pair<int32_t, int64_t>> ent;
    for (int32_t i = 0; i < M->m; ++i) {
        ent.clear();
        for (int64_t p = cnt[i]; p < cnt[i + 1]; ++p) ent.emplace_back(col[p], p);
        std::stable_sort(ent.begin(), ent.end(),
                         [](const std::pair<int32_t, int64_t>& a, const std::pair<int32_t, int64_t>& b) {
                             return a.first < b.first;
                         });
        for (size_t e = 0; e < ent.size(); ++e) {
            if (e > 0 && ent[e].first == ent[e - 1].first) {
                M->v.back() += val[ent[e].second];
            } else {
                M->ci.push_back(ent[e].first);
                M->v.push_back(val[ent[e].second]);
            }
        }
        M->rp[i + 1] = static_cast<int32_t>(M->ci.size());
    }
    return M.release();
}

void mps_destroy(MpsModel* m) { delete m; }

}  // namespace pdfp
