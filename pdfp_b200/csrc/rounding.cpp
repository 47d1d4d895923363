// rounding.cpp -- the pump's constraint-propagation rounding on the host, native.
//
// FP 2.0's CPR rounding as the reference runs it on the CPU: activity-based bound
// propagation (src/propagation.jl:1-276) driving a guarded two-phase rounding
// (src/rounding.jl:117-256).  Everything that depends only on the model is built
// once per pump run (Rounder); each rounding call starts fresh domains, fixes the
// integer columns in the order the caller ranked them, propagates after each fix
// (phase one, and phase three) or once after a whole batch of already-integral
// columns (phase two, the guard: the caller discards the call when the batch makes
// the domains infeasible).  The ranking, its random swaps and the batch policy stay
// with the caller.  Arithmetic is plain IEEE double in the reference's order (built
// with -ffp-contract=off), so the results equal an exact restatement bit for bit.
#include <cmath>
#include <cstdint>
#include <deque>
#include <vector>

#include "../../include/pdfp_b200.h"
#include "device.hpp"
#include "solvers.hpp"

namespace pdfp {
namespace {

constexpr double kBoundTol = 1e-6;       // src/propagation.jl:7
constexpr double kInfeasTol = 1e-6;      // :8
constexpr int kMaxTightenings = 10;      // :9
constexpr double kDomainInfinity = 1e12; // :10
enum RowKind : int8_t { kGeneral = 0, kCardinality = 1, kKnapsack = 2 };  // :14-16

// Julia round on a Float64: nearest, ties to even (the default rounding mode).
inline double jround(double v) { return std::nearbyint(v); }
inline double clampv(double x, double lo, double hi) { return x > hi ? hi : (x < lo ? lo : x); }

}  // namespace

// The model part (src/propagation.jl:19-84).
struct Rounder {
    int32_t m = 0, n = 0;
    std::vector<int32_t> cp, cr;  // CSC: column pointers, row indices (ascending)
    std::vector<double> cv;
    std::vector<int32_t> rp, rc;  // CSR: row pointers, column indices (ascending)
    std::vector<double> rv;
    std::vector<double> b, l, u, L_min, L_max, row_maxcoef, row_maxroom;
    std::vector<uint8_t> is_le, is_int;
    std::vector<int8_t> row_kind;
};

namespace {

// Domains of one rounding call and the propagation queue (src/propagation.jl:87-107).
struct State {
    const Rounder& d;
    std::vector<double> l, u, L_min, L_max, row_maxroom;
    std::vector<uint8_t> in_queue;
    std::deque<int32_t> queue;
    std::vector<int32_t> tighten_lo, tighten_hi;
    int64_t max_pops;
    bool infeasible = false;

    State(const Rounder& r, int64_t pops)
        : d(r), l(r.l), u(r.u), L_min(r.L_min), L_max(r.L_max), row_maxroom(r.row_maxroom),
          in_queue(r.m, 0), tighten_lo(r.n, 0), tighten_hi(r.n, 0), max_pops(pops) {}

    void enqueue(int32_t i) {
        if (!in_queue[i]) {
            queue.push_back(i);
            in_queue[i] = 1;
        }
    }
    bool fixed(int32_t j) const { return std::fabs(u[j] - l[j]) < kBoundTol; }

    bool tighten_upper(int32_t j, double new_u) {  // src/propagation.jl:117-136
        const double u_old = u[j];
        if (!(new_u < u_old - kBoundTol)) return false;
        double nu = d.is_int[j] ? std::floor(new_u + kBoundTol) : new_u;
        if (nu < l[j] - kBoundTol) nu = l[j];
        if (l[j] > nu) nu = l[j];
        if (nu >= u_old - kBoundTol) return false;
        u[j] = nu;
        tighten_hi[j] += 1;
        const bool wake = tighten_hi[j] <= kMaxTightenings || std::fabs(nu - l[j]) < kBoundTol;
        const double du = nu - u_old;
        for (int32_t k = d.cp[j]; k < d.cp[j + 1]; ++k) {
            const int32_t i = d.cr[k];
            const double a = d.cv[k];
            if (a > 0) L_max[i] += a * du; else L_min[i] += a * du;
            if (wake) enqueue(i);
        }
        return true;
    }

    bool tighten_lower(int32_t j, double new_l) {  // src/propagation.jl:138-156
        const double l_old = l[j];
        if (!(new_l > l_old + kBoundTol)) return false;
        double nl = d.is_int[j] ? std::ceil(new_l - kBoundTol) : new_l;
        if (nl > u[j] + kBoundTol) nl = u[j];
        if (u[j] < nl) nl = u[j];
        if (nl <= l_old + kBoundTol) return false;
        l[j] = nl;
        tighten_lo[j] += 1;
        const bool wake = tighten_lo[j] <= kMaxTightenings || std::fabs(u[j] - nl) < kBoundTol;
        const double dl = nl - l_old;
        for (int32_t k = d.cp[j]; k < d.cp[j + 1]; ++k) {
            const int32_t i = d.cr[k];
            const double a = d.cv[k];
            if (a > 0) L_min[i] += a * dl; else L_max[i] += a * dl;
            if (wake) enqueue(i);
        }
        return true;
    }

    void cardinality_row(int32_t i) {  // src/propagation.jl:160-177
        const bool is_eq = !d.is_le[i];
        const double slack_up = d.b[i] - L_min[i];
        const double slack_dn = L_max[i] - d.b[i];
        if (slack_up < -kInfeasTol || (is_eq && slack_dn < -kInfeasTol)) {
            infeasible = true;
            return;
        }
        const bool up = slack_up < 1.0 - kBoundTol;
        const bool dn = is_eq && slack_dn < 1.0 - kBoundTol;
        if (!(up || dn)) return;
        for (int32_t k = d.rp[i]; k < d.rp[i + 1]; ++k) {
            const int32_t j = d.rc[k];
            if (up) tighten_upper(j, l[j] + slack_up);
            if (dn) tighten_lower(j, u[j] - slack_dn);
        }
    }

    void knapsack_row(int32_t i) {  // src/propagation.jl:180-192
        const double slack_up = d.b[i] - L_min[i];
        if (slack_up < -kInfeasTol) {
            infeasible = true;
            return;
        }
        if (d.row_maxcoef[i] <= slack_up + kBoundTol) return;
        for (int32_t k = d.rp[i]; k < d.rp[i + 1]; ++k)
            if (d.rv[k] > slack_up + kBoundTol) tighten_upper(d.rc[k], l[d.rc[k]]);
    }

    void row(int32_t i) {  // src/propagation.jl:194-232
        if (d.row_kind[i] == kCardinality) return cardinality_row(i);
        if (d.row_kind[i] == kKnapsack) return knapsack_row(i);
        const bool is_le = d.is_le[i] != 0;
        const double slack_up = d.b[i] - L_min[i];
        const double slack_dn = L_max[i] - d.b[i];
        if (slack_up < -kInfeasTol || (!is_le && slack_dn < -kInfeasTol)) {
            infeasible = true;
            return;
        }
        const double threshold = (is_le ? slack_up : (slack_dn < slack_up ? slack_dn : slack_up)) + kBoundTol;
        if (row_maxroom[i] <= threshold) return;
        double max_room = 0.0;
        for (int32_t k = d.rp[i]; k < d.rp[i + 1]; ++k) {
            const int32_t j = d.rc[k];
            const double room = std::fabs(d.rv[k]) * (u[j] - l[j]);
            if (room > max_room) max_room = room;
        }
        row_maxroom[i] = max_room;
        if (is_le && max_room <= slack_up + kBoundTol) return;
        for (int32_t k = d.rp[i]; k < d.rp[i + 1]; ++k) {
            const int32_t j = d.rc[k];
            const double a = d.rv[k];
            if (a > 0) tighten_upper(j, l[j] + slack_up / a);
            else tighten_lower(j, u[j] + slack_up / a);
            if (!is_le) {
                if (a > 0) tighten_lower(j, u[j] - slack_dn / a);
                else tighten_upper(j, l[j] - slack_dn / a);
            }
        }
    }

    void propagate() {  // src/propagation.jl:235-244
        int64_t pops = 0;
        while (!queue.empty() && pops < max_pops) {
            const int32_t i = queue.front();
            queue.pop_front();
            in_queue[i] = 0;
            row(i);
            ++pops;
        }
    }

    bool fix(int32_t j, double value) {  // src/propagation.jl:252-274
        if (value < l[j] - kBoundTol || value > u[j] + kBoundTol) {
            infeasible = true;
            return false;
        }
        const double lo = l[j], hi = u[j];
        const double v = value > hi ? hi : (value < lo ? lo : value);
        if (std::fabs(v - lo) < kBoundTol && std::fabs(v - hi) < kBoundTol) return true;
        l[j] = v;
        u[j] = v;
        tighten_lo[j] += 1;
        tighten_hi[j] += 1;
        const double dl = v - lo, du = v - hi;
        for (int32_t k = d.cp[j]; k < d.cp[j + 1]; ++k) {
            const int32_t i = d.cr[k];
            const double a = d.cv[k];
            if (a > 0) {
                L_min[i] += a * dl;
                L_max[i] += a * du;
            } else {
                L_min[i] += a * du;
                L_max[i] += a * dl;
            }
            enqueue(i);
        }
        return true;
    }
};

// src/rounding.jl:117-118
inline double row_violation(const Rounder& d, int32_t i, double activity) {
    const double e = activity - d.b[i];
    return d.is_le[i] ? (e > 0.0 ? e : 0.0) : std::fabs(e);
}

// Violation-guided rounding (src/rounding.jl:123-141).
double guided_value(const State& s, int32_t j, double target, const std::vector<double>& act) {
    if (!(s.u[j] - s.l[j] > kBoundTol)) return target;
    const double lo = std::ceil(s.l[j] - kBoundTol);
    const double hi = std::floor(s.u[j] + kBoundTol);
    if (!(hi > lo)) return target;
    const Rounder& d = s.d;
    auto score = [&](double v) {
        double t = 0.0;
        for (int32_t k = d.cp[j]; k < d.cp[j + 1]; ++k) {
            const int32_t i = d.cr[k];
            t += row_violation(d, i, act[i] + d.cv[k] * v) - row_violation(d, i, act[i]);
        }
        return t;
    };
    const double score_lo = score(lo), score_hi = score(hi);
    if (score_lo < score_hi - 1e-12) return lo;
    if (score_hi < score_lo - 1e-12) return hi;
    return target;
}

void add_activity(const Rounder& d, std::vector<double>& act, int32_t j, double v) {
    for (int32_t k = d.cp[j]; k < d.cp[j + 1]; ++k) act[d.cr[k]] += d.cv[k] * v;
}

// src/rounding.jl:152-174
void round_sequentially(State& s, double* xt, const int32_t* idx, int32_t count, const double* xs,
                        const uint8_t* direction, std::vector<double>& act) {
    for (int32_t t = 0; t < count; ++t) {
        const int32_t j = idx[t];
        if (s.fixed(j)) {
            xt[j] = s.l[j];
            continue;
        }
        double target = jround(clampv(xs[j], s.l[j], s.u[j]));
        if (target < s.l[j] - kBoundTol || target > s.u[j] + kBoundTol) {
            const double other = jround(clampv(xs[j] + (target < s.l[j] ? 1.0 : -1.0), s.l[j], s.u[j]));
            target = clampv(other, s.l[j], s.u[j]);
        }
        if (direction && direction[j]) target = guided_value(s, j, target, act);
        s.fix(j, target);
        s.propagate();
        if (direction) add_activity(s.d, act, j, target);
        xt[j] = target;
    }
}

}  // namespace

Rounder* rounder_create(const pdfp_csr* A, const double* b, const uint8_t* is_le, const double* l,
                        const double* u, const uint8_t* is_int) {
    auto r = new Rounder();
    const int32_t m = A->m, n = A->n;
    r->m = m;
    r->n = n;
    const int64_t nnz = m > 0 ? A->row_ptr[m] : 0;
    r->rp.assign(A->row_ptr, A->row_ptr + m + 1);
    r->rc.assign(A->col_idx, A->col_idx + nnz);
    r->rv.assign(A->val, A->val + nnz);
    for (int32_t i = 0; i < m; ++i)
        for (int32_t k = r->rp[i] + 1; k < r->rp[i + 1]; ++k)
            if (r->rc[k] <= r->rc[k - 1]) {
                delete r;
                throw Error(E_INVALID, "rounder: column indices must ascend within each row");
            }
    for (int64_t k = 0; k < nnz; ++k)
        if (r->rc[k] < 0 || r->rc[k] >= n) {
            delete r;
            throw Error(E_INVALID, "rounder: column index out of range");
        }
    // CSC by a counting pass: rows come out ascending within each column
    r->cp.assign(n + 1, 0);
    for (int64_t k = 0; k < nnz; ++k) r->cp[r->rc[k] + 1] += 1;
    for (int32_t j = 0; j < n; ++j) r->cp[j + 1] += r->cp[j];
    r->cr.resize(nnz);
    r->cv.resize(nnz);
    std::vector<int32_t> next(r->cp.begin(), r->cp.end() - 1);
    for (int32_t i = 0; i < m; ++i)
        for (int32_t k = r->rp[i]; k < r->rp[i + 1]; ++k) {
            const int32_t p = next[r->rc[k]]++;
            r->cr[p] = i;
            r->cv[p] = r->rv[k];
        }
    r->b.assign(b, b + m);
    r->is_le.assign(is_le, is_le + m);
    r->is_int.assign(is_int, is_int + n);
    r->l.resize(n);
    r->u.resize(n);
    for (int32_t j = 0; j < n; ++j) {
        r->l[j] = std::isfinite(l[j]) ? l[j] : -kDomainInfinity;
        r->u[j] = std::isfinite(u[j]) ? u[j] : kDomainInfinity;
    }
    r->L_min.assign(m, 0.0);
    r->L_max.assign(m, 0.0);
    r->row_kind.assign(m, kGeneral);
    r->row_maxcoef.assign(m, 0.0);
    r->row_maxroom.assign(m, 0.0);
    for (int32_t i = 0; i < m; ++i) {
        double lmin = 0.0, lmax = 0.0;
        for (int32_t k = r->rp[i]; k < r->rp[i + 1]; ++k) {
            const int32_t j = r->rc[k];
            const double a = r->rv[k];
            if (a > 0) {
                lmin += a * r->l[j];
                lmax += a * r->u[j];
            } else {
                lmin += a * r->u[j];
                lmax += a * r->l[j];
            }
        }
        r->L_min[i] = lmin;
        r->L_max[i] = lmax;
        bool all_one = true, all_pos = true, all_bin = true;
        double maxcoef = 0.0;
        for (int32_t k = r->rp[i]; k < r->rp[i + 1]; ++k) {
            const int32_t j = r->rc[k];
            const double a = r->rv[k];
            if (std::fabs(a) > maxcoef) maxcoef = std::fabs(a);
            if (a != 1.0) all_one = false;
            if (!(a > 0.0)) all_pos = false;
            if (!(r->is_int[j] && l[j] == 0.0 && u[j] == 1.0)) all_bin = false;
            if (!(all_bin && (all_one || all_pos))) break;
        }
        r->row_maxcoef[i] = maxcoef;
        if (all_bin && all_one) r->row_kind[i] = kCardinality;
        else if (all_bin && all_pos && r->is_le[i]) r->row_kind[i] = kKnapsack;
        double room = 0.0;
        for (int32_t k = r->rp[i]; k < r->rp[i + 1]; ++k) {
            const int32_t j = r->rc[k];
            const double width = u[j] - l[j];
            const double rr = std::isfinite(width) ? std::fabs(r->rv[k]) * width : INFINITY;
            if (rr > room) room = rr;
        }
        r->row_maxroom[i] = room;
    }
    return r;
}

void rounder_destroy(Rounder* r) { delete r; }

// One rounding call; see pdfp_rounder_round.
void rounder_round(const Rounder& r, const double* xs, const int32_t* first, int32_t n_first,
                   int32_t batch_phase, const int32_t* batch, int32_t n_batch, const int32_t* after,
                   int32_t n_after, const int32_t* int_idx, int32_t n_int, const uint8_t* direction,
                   int64_t max_pops, double* xt, int32_t* infeasible) {
    auto check = [&](const int32_t* idx, int32_t cnt) {
        for (int32_t t = 0; t < cnt; ++t)
            if (idx[t] < 0 || idx[t] >= r.n) throw Error(E_INVALID, "rounder: column index out of range");
    };
    check(first, n_first);
    check(batch, n_batch);
    check(after, n_after);
    check(int_idx, n_int);
    if (max_pops < 0) throw Error(E_INVALID, "rounder: max_pops must be >= 0");
    State s(r, max_pops);
    std::vector<double> act(direction ? r.m : 0, 0.0);
    for (int32_t j = 0; j < r.n; ++j) xt[j] = xs[j];
    round_sequentially(s, xt, first, n_first, xs, direction, act);
    if (batch_phase) {
        for (int32_t t = 0; t < n_batch; ++t) {
            const int32_t j = batch[t];
            if (s.fixed(j)) {
                xt[j] = s.l[j];
                continue;
            }
            const double target = jround(clampv(xs[j], s.l[j], s.u[j]));
            s.fix(j, target);
            if (direction) add_activity(r, act, j, target);
            xt[j] = target;
        }
        s.propagate();
        if (s.infeasible) {  // the guard: the caller discards this call
            *infeasible = 2;
            return;
        }
    }
    round_sequentially(s, xt, after, n_after, xs, direction, act);
    for (int32_t t = 0; t < n_int; ++t) {  // the integers as the domains leave them
        const int32_t j = int_idx[t];
        xt[j] = s.fixed(j) ? s.l[j] : jround(clampv(xs[j], s.l[j], s.u[j]));
    }
    *infeasible = s.infeasible ? 1 : 0;
}

}  // namespace pdfp
