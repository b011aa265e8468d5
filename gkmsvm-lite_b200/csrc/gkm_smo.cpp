// gkm_smo.cpp -- host SMO solver for gkm-SVM training (C-SVC and epsilon-SVR),
// taking kernel columns from a caller's provider (solver.py:13-392 and
// _csmo.c of gkmsvm-lite; its column provider here is the GPU l-mer index).
//
// The dual, as LIBSVM states it: minimise 1/2 a'Qa + p'a subject to y'a = 0
// and 0 <= a_t <= C_t, with Q_ts = y_t y_s K(t mod N, s mod N) over n dual
// variables of N sequences (n = N for C-SVC, p = -1; n = 2N for SVR, signs
// +1 then -1, p = (eps - z, eps + z)).  Each iteration picks a working pair by
// second-order selection (WSS3 of Fan, Chen and Lin, JMLR 2005), solves the
// two-variable problem analytically with clipping to the box, and updates the
// gradient G = Qa + p with the two columns.  It stops when the maximal KKT
// violation m(a) - M(a) is below tol.  The bias is -rho, rho the mean of
// y_t G_t over free variables (or the midpoint of its bounds).
//
// Shrinking (the method of LIBSVM, Chang and Lin): every min(n, 1000)
// iterations the variables at a bound whose gradient says they will stay
// there leave the active set, and selection and gradient updates run over the
// active set only.  G_bar_t = sum over variables at their upper bound of
// C_s Q_ts is kept up to date (a column per bound change), so the gradient of
// the inactive variables can be rebuilt from G_bar, p and the free variables'
// columns: once when the violation first falls below 10 tol (then every
// variable is active again and shrinking resumes), and when the active set
// has converged, before the final check over all variables.
//
// Columns: an LRU cache of cache_columns columns of N doubles.  On a miss
// the solver asks the provider for the column and, while the cache has free
// slots, for up to prefetch - 1 more: the sequences of the variables most
// likely to join the next working sets (the ends of -y G in the up and low
// sets), so a GPU provider answers a batch per call.
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <list>
#include <unordered_map>
#include <vector>

#include "gkm_b200.h"

int gkm_fail(int code, const char *fmt, ...);

namespace {

constexpr double TAU = 1e-12;
constexpr double INF = std::numeric_limits<double>::infinity();

class ColumnCache {
  public:
    ColumnCache(int N, int capacity, gkm_columns_cb cb, void *ctx)
        : N_(N), cap_(std::max(2, std::min(capacity, N))), cb_(cb), ctx_(ctx)
    {
    }

    bool cached(int c) const { return where_.count(c) != 0; }
    int free_slots() const { return cap_ - (int)where_.size(); }

    // column c (length N), fetched with `extra` (not cached, distinct) when missing;
    // nullptr if the provider failed
    const double *get(int c, const std::vector<int> &extra)
    {
        auto it = where_.find(c);
        if (it != where_.end()) {
            lru_.splice(lru_.begin(), lru_, it->second.pos);
            return it->second.data.data();
        }
        std::vector<int32_t> req{c};
        for (int e : extra)
            if ((int)req.size() < free_slots() && !cached(e) && e != c) req.push_back(e);
        std::vector<double> buf((size_t)req.size() * N_);
        if (cb_((int32_t)req.size(), req.data(), buf.data(), ctx_) != 0) return nullptr;
        calls_++;
        const double *out = nullptr;
        for (size_t k = 0; k < req.size(); k++) {
            if (k > 0 && free_slots() <= 0) break;
            if (free_slots() <= 0) evict();
            Entry &e = where_[req[k]];
            e.data.assign(buf.begin() + k * N_, buf.begin() + (k + 1) * N_);
            lru_.push_front(req[k]);
            e.pos = lru_.begin();
            if (k == 0) out = e.data.data();
            else prefetched_++;
        }
        // the requested column goes to the front (it was inserted first)
        lru_.splice(lru_.begin(), lru_, where_[c].pos);
        return out;
    }

    // pins: the solver holds two columns at once; they are the two most recent
    void evict()
    {
        const int c = lru_.back();
        lru_.pop_back();
        where_.erase(c);
    }

    int64_t calls_ = 0, prefetched_ = 0;

  private:
    struct Entry {
        std::vector<double> data;
        std::list<int>::iterator pos;
    };
    int N_, cap_;
    gkm_columns_cb cb_;
    void *ctx_;
    std::list<int> lru_;
    std::unordered_map<int, Entry> where_;
};

struct Solver {
    int n, N;
    const double *y, *p, *diag;
    double Cp, Cn, tol;
    std::vector<double> a, G, G_bar;
    std::vector<int> active;  // the active variables, ascending
    bool unshrunk = false;    // the one rebuild at 10 tol has happened
    ColumnCache cache;
    int prefetch;

    Solver(int n_, int N_, const double *y_, const double *p_, const double *diag_, double Cp_, double Cn_,
           double tol_, int cache_columns, int prefetch_, gkm_columns_cb cb, void *ctx)
        : n(n_), N(N_), y(y_), p(p_), diag(diag_), Cp(Cp_), Cn(Cn_), tol(tol_), a(n_, 0.0), G(p_, p_ + n_),
          G_bar(n_, 0.0), active(n_), cache(N_, cache_columns, cb, ctx), prefetch(prefetch_)
    {
        for (int t = 0; t < n; t++) active[t] = t;
    }

    double C(int t) const { return y[t] > 0 ? Cp : Cn; }
    bool upper(int t) const { return a[t] >= C(t); }
    bool lower(int t) const { return a[t] <= 0.0; }
    bool in_up(int t) const { return y[t] > 0 ? !upper(t) : !lower(t); }
    bool in_low(int t) const { return y[t] > 0 ? !lower(t) : !upper(t); }
    double Kdiag(int t) const { return diag ? diag[t % N] : 1.0; }

    // sequences of the likeliest next working-set variables, not cached
    std::vector<int> candidates(int skip) const
    {
        std::vector<int> out;
        const int k = std::min(prefetch - 1, cache.free_slots() - 1);
        if (k <= 0) return out;
        std::vector<std::pair<double, int>> up, low;
        for (int t : active) {
            const int c = t % N;
            if (c == skip || cache.cached(c)) continue;
            const double s = -y[t] * G[t];
            if (in_up(t)) up.push_back({-s, c});   // largest -y G first
            if (in_low(t)) low.push_back({s, c});  // smallest -y G first
        }
        const int half = std::max(1, k / 2);
        for (auto *v : {&up, &low}) {
            const int take = std::min<int>(half, (int)v->size());
            if (take == 0) continue;
            std::partial_sort(v->begin(), v->begin() + take, v->end());
            for (int q = 0; q < take; q++) out.push_back((*v)[q].second);
        }
        std::sort(out.begin(), out.end());
        out.erase(std::unique(out.begin(), out.end()), out.end());
        if ((int)out.size() > k) out.resize(k);
        return out;
    }

    const double *column(int t)
    {
        const int c = t % N;
        return cache.get(c, cache.cached(c) ? std::vector<int>() : candidates(c));
    }

    // WSS3; false when optimal (or no pair)
    int select(int &oi, int &oj, const double *&Ki, bool &failed)
    {
        double Gmax = -INF, Gmax2 = -INF, best = INF;
        int i = -1, j = -1;
        for (int t : active) {
            if (!in_up(t)) continue;
            const double v = -y[t] * G[t];
            if (v >= Gmax) {
                Gmax = v;
                i = t;
            }
        }
        if (i < 0) return 0;
        Ki = column(i);
        if (!Ki) {
            failed = true;
            return 0;
        }
        for (int t : active) {
            if (!in_low(t)) continue;
            const double v = -y[t] * G[t];
            if (-v >= Gmax2) Gmax2 = -v;
            const double b = Gmax - v;
            if (b > 0) {
                // second-order gain: the pair's curvature Q_ii + Q_tt - 2 y_i y_t Q_it
                // = K_ii + K_tt - 2 K_it (Q_it = y_i y_t K_it)
                double q = Kdiag(i) + Kdiag(t) - 2.0 * Ki[t % N];
                if (q <= 0) q = TAU;
                const double obj = -(b * b) / q;
                if (obj <= best) {
                    best = obj;
                    j = t;
                }
            }
        }
        if (Gmax + Gmax2 < tol || j < 0) return 0;
        oi = i;
        oj = j;
        return 1;
    }

    // G_t for the inactive t from G_bar, p and the free variables' columns
    // (inactive variables sit at a bound, so every free one is active);
    // false if the provider failed
    bool reconstruct()
    {
        if ((int)active.size() == n) return true;
        std::vector<char> act(n, 0);
        for (int t : active) act[t] = 1;
        std::vector<int> idle;
        for (int t = 0; t < n; t++)
            if (!act[t]) {
                idle.push_back(t);
                G[t] = G_bar[t] + p[t];
            }
        for (int j : active) {
            if (upper(j) || lower(j)) continue;
            const double *Kj = column(j);
            if (!Kj) return false;
            const double c = y[j] * a[j];
            for (int t : idle) G[t] += y[t] * c * Kj[t % N];
        }
        return true;
    }

    void activate_all()
    {
        active.resize(n);
        for (int t = 0; t < n; t++) active[t] = t;
    }

    // drop the variables that will stay at their bound; false if the
    // provider failed during the one rebuild
    bool shrink()
    {
        double m = -INF, M = -INF;  // max over up of -y G, max over low of y G
        for (int t : active) {
            if (in_up(t)) m = std::max(m, -y[t] * G[t]);
            if (in_low(t)) M = std::max(M, y[t] * G[t]);
        }
        if (!unshrunk && m + M <= 10.0 * tol) {
            unshrunk = true;
            if (!reconstruct()) return false;
            activate_all();
        }
        std::vector<int> keep;
        keep.reserve(active.size());
        for (int t : active) {
            bool drop = false;
            if (upper(t))
                drop = y[t] > 0 ? -G[t] > m : -G[t] > M;
            else if (lower(t))
                drop = y[t] > 0 ? G[t] > M : G[t] > m;
            if (!drop) keep.push_back(t);
        }
        active.swap(keep);
        return true;
    }

    // keep G_bar up to date for a variable whose upper-bound status changed;
    // Kt its column
    void bound_change(int t, bool was_upper, const double *Kt)
    {
        if (was_upper == upper(t)) return;
        const double c = (was_upper ? -1.0 : 1.0) * C(t) * y[t];
        for (int s = 0; s < n; s++) G_bar[s] += c * y[s] * Kt[s % N];
    }

    double rho() const
    {
        double ub = INF, lb = -INF, sum = 0.0;
        int nfree = 0;
        for (int t = 0; t < n; t++) {
            const double yG = y[t] * G[t];
            if (upper(t)) {
                if (y[t] < 0) ub = std::min(ub, yG);
                else lb = std::max(lb, yG);
            } else if (lower(t)) {
                if (y[t] > 0) ub = std::min(ub, yG);
                else lb = std::max(lb, yG);
            } else {
                nfree++;
                sum += yG;
            }
        }
        return nfree > 0 ? sum / nfree : (ub + lb) / 2;
    }
};

}  // namespace

extern "C" int gkm_smo_solve(int32_t n, int32_t N, const double *y, const double *p, const double *diag,
                             double C_pos, double C_neg, double tol, int64_t max_iter, int32_t cache_columns,
                             int32_t prefetch, gkm_columns_cb columns, void *ctx, double *coef, double *bias,
                             int64_t *iterations, int32_t verbose)
{
    if (!y || !p || !columns || !coef || !bias) return gkm_fail(GKM_ERR_INVALID, "null argument");
    if (N < 1 || n < 1 || n % N != 0) return gkm_fail(GKM_ERR_INVALID, "n (%d) must be a multiple of N (%d)", n, N);
    if (!(C_pos > 0) || !(C_neg > 0) || !(tol > 0)) return gkm_fail(GKM_ERR_INVALID, "C and tol must be positive");
    for (int t = 0; t < n; t++)
        if (y[t] != 1.0 && y[t] != -1.0) return gkm_fail(GKM_ERR_INVALID, "signs must be +1 or -1");
    Solver s(n, N, y, p, diag, C_pos, C_neg, tol, cache_columns, std::max(1, prefetch), columns, ctx);
    int64_t it = 0;
    bool failed = false;
    int counter = std::min(n, 1000) + 1;
    for (; it < max_iter; it++) {
        if (--counter == 0) {
            counter = std::min(n, 1000);
            if (!s.shrink()) {
                failed = true;
                break;
            }
        }
        int i = -1, j = -1;
        const double *Ki = nullptr;
        if (!s.select(i, j, Ki, failed)) {
            // converged on the active set: check every variable
            if (failed || (int)s.active.size() == n) break;
            if (!s.reconstruct()) {
                failed = true;
                break;
            }
            s.activate_all();
            if (!s.select(i, j, Ki, failed)) break;
            counter = 1;
        }
        // Ki stays valid: fetching j evicts only the least recently used column
        // and i's was used last
        const double *Kj = s.column(j);
        if (!Kj) {
            failed = true;
            break;
        }
        Ki = s.column(i);  // i's column again (a hit; its storage did not move)
        const double Ci = s.C(i), Cj = s.C(j);
        const double ai0 = s.a[i], aj0 = s.a[j];
        const bool ui = s.upper(i), uj = s.upper(j);
        double &ai = s.a[i], &aj = s.a[j];
        const double Kij = Ki[j % N];
        const double yi = y[i], yj = y[j];
        // the pair's curvature along the feasible direction: K_ii + K_jj - 2 K_ij
        // for either sign combination
        if (yi != yj) {
            double q = s.Kdiag(i) + s.Kdiag(j) - 2.0 * Kij;
            if (q <= 0) q = TAU;
            const double delta = (-s.G[i] - s.G[j]) / q, diff = ai - aj;
            ai += delta;
            aj += delta;
            if (diff > 0) {
                if (aj < 0) {
                    aj = 0;
                    ai = diff;
                }
            } else if (ai < 0) {
                ai = 0;
                aj = -diff;
            }
            if (diff > Ci - Cj) {
                if (ai > Ci) {
                    ai = Ci;
                    aj = Ci - diff;
                }
            } else if (aj > Cj) {
                aj = Cj;
                ai = Cj + diff;
            }
        } else {
            double q = s.Kdiag(i) + s.Kdiag(j) - 2.0 * Kij;
            if (q <= 0) q = TAU;
            const double delta = (s.G[i] - s.G[j]) / q, sum = ai + aj;
            ai -= delta;
            aj += delta;
            if (sum > Ci) {
                if (ai > Ci) {
                    ai = Ci;
                    aj = sum - Ci;
                }
            } else if (aj < 0) {
                aj = 0;
                ai = sum;
            }
            if (sum > Cj) {
                if (aj > Cj) {
                    aj = Cj;
                    ai = sum - Cj;
                }
            } else if (ai < 0) {
                ai = 0;
                aj = sum;
            }
        }
        const double dai = ai - ai0, daj = aj - aj0;
        // G_t += Q_ti dai + Q_tj daj, Q_ts = y_t y_s K(t mod N, s mod N)
        const double ci = yi * dai, cj = yj * daj;
        for (int t : s.active) s.G[t] += y[t] * (ci * Ki[t % N] + cj * Kj[t % N]);
        s.bound_change(i, ui, Ki);
        s.bound_change(j, uj, Kj);
        if (verbose && (it + 1) % 100000 == 0)
            fprintf(stderr, "  SMO iteration %lld\n", (long long)(it + 1));
    }
    if (!failed && !s.reconstruct()) failed = true;  // stopped by max_iter with variables shrunk
    if (failed) return gkm_fail(GKM_ERR_INVALID, "the kernel column provider failed");
    for (int t = 0; t < n; t++) coef[t] = y[t] * s.a[t];
    *bias = -s.rho();
    if (iterations) *iterations = it;
    if (verbose)
        fprintf(stderr, "  SMO: %lld iterations, %lld column calls, %lld columns prefetched\n", (long long)it,
                (long long)s.cache.calls_, (long long)s.cache.prefetched_);
    return GKM_OK;
}
