// C ABI over the host CMA-ES (include/ta3b_cma.h).
#include "../../include/ta3b_cma.h"

#include "cmaes.hpp"

#include <cmath>
#include <cstring>
#include <memory>
#include <string>

using namespace ta3b::host;

struct ta3c_opt {
    std::unique_ptr<Cma> cma;
};

namespace {
thread_local std::string g_err;

int fail(char const* msg) {
    g_err = msg;
    return 1;
}

// test_problems.hpp:49-73: a fixed rotation from mt19937(0xdd) normal draws,
// orthonormalised (modified Gram-Schmidt over the columns)
Mat rotation(int n) {
    std::mt19937 rng(0xdd);
    std::normal_distribution<double> nd(0.0, 1.0);
    Mat m(n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) m(i, j) = nd(rng);
    for (int c = 0; c < n; ++c) {
        for (int p = 0; p < c; ++p) {
            double d = 0.0;
            for (int r = 0; r < n; ++r) d += m(r, c) * m(r, p);
            for (int r = 0; r < n; ++r) m(r, c) -= d * m(r, p);
        }
        double s = 0.0;
        for (int r = 0; r < n; ++r) s += m(r, c) * m(r, c);
        s = std::sqrt(s);
        for (int r = 0; r < n; ++r) m(r, c) /= s;
    }
    return m;
}

double ellipsoid(double const* x, int n) {
    double sum = 0.0;
    for (int i = 0; i < n; ++i) sum += std::pow(1e6, double(i) / (double(n) - 1.0)) * x[i] * x[i];
    return sum;
}
} // namespace

extern "C" {

ta3c_opt* ta3c_create(int kind, uint32_t dim, const double* x0, const double* lb, const double* ub, double sigma0,
                      uint32_t seed, int active_update) {
    if (dim == 0 || !x0 || !lb || !ub) {
        fail("ta3c_create: dim must be positive and x0 / lb / ub non-null");
        return nullptr;
    }
    if (!(sigma0 > 0.0)) {
        fail("ta3c_create: sigma0 must be positive");
        return nullptr;
    }
    for (uint32_t j = 0; j < dim; ++j)
        if (!std::isfinite(lb[j]) || !std::isfinite(ub[j])) {
            fail("ta3c_create: finite box bounds required");
            return nullptr;
        }
    vec const x(x0, x0 + dim), l(lb, lb + dim), u(ub, ub + dim);
    auto* o = new ta3c_opt;
    if (kind == TA3C_SEP)
        o->cma.reset(new SepCma(x, l, u, sigma0, seed));
    else if (kind == TA3C_DD)
        o->cma.reset(new DdCma(x, l, u, sigma0, seed, active_update != 0));
    else {
        delete o;
        fail("ta3c_create: kind must be TA3C_SEP or TA3C_DD");
        return nullptr;
    }
    return o;
}

void ta3c_destroy(ta3c_opt* opt) { delete opt; }

int ta3c_new_evolve(ta3c_opt* opt) {
    if (!opt) return fail("null optimiser");
    opt->cma->new_evolve();
    return 0;
}

int ta3c_ask(ta3c_opt* opt, uint32_t lam, double* x_out) {
    if (!opt || !x_out) return fail("ta3c_ask: null argument");
    if (lam < 5) return fail("ta3c_ask: at least 5 candidates per generation");
    opt->cma->ask(int(lam), x_out);
    return 0;
}

double ta3c_last_dx(const ta3c_opt* opt) { return opt ? opt->cma->last_dx() : 0.0 / 0.0; }

int ta3c_tell(ta3c_opt* opt, uint32_t k, const int32_t* idx, const double* fitness) {
    if (!opt || !fitness) return fail("ta3c_tell: null argument");
    if (k < 5) return fail("ta3c_tell: at least 5 evaluated candidates");
    int const asked = opt->cma->asked();
    if (int64_t(k) > asked) return fail("ta3c_tell: more fitness values than asked candidates");
    if (idx)
        for (uint32_t j = 0; j < k; ++j)
            if (idx[j] < 0 || idx[j] >= asked) return fail("ta3c_tell: candidate index out of range");
    opt->cma->tell(int(k), idx, fitness);
    return 0;
}

int ta3c_mean(const ta3c_opt* opt, double* out) {
    if (!opt || !out) return fail("ta3c_mean: null argument");
    vec const& m = opt->cma->mean();
    std::memcpy(out, m.data(), m.size() * sizeof(double));
    return 0;
}

double ta3c_sigma(const ta3c_opt* opt) { return opt ? opt->cma->sigma() : 0.0 / 0.0; }

int ta3c_axis_std(const ta3c_opt* opt, double* out) {
    if (!opt || !out) return fail("ta3c_axis_std: null argument");
    vec const s = opt->cma->axis_std();
    std::memcpy(out, s.data(), s.size() * sizeof(double));
    return 0;
}

int ta3c_whiten(const ta3c_opt* opt, uint32_t k, const double* x, double* z_out) {
    if (!opt || (k && (!x || !z_out))) return fail("ta3c_whiten: null argument");
    opt->cma->whiten(int(k), x, z_out);
    return 0;
}

uint32_t ta3c_dim(const ta3c_opt* opt) { return opt ? uint32_t(opt->cma->dim()) : 0u; }

uint64_t ta3c_save(const ta3c_opt* opt, void* buf, uint64_t cap) {
    if (!opt) return 0;
    std::string const s = opt->cma->save();
    if (buf && cap >= s.size()) std::memcpy(buf, s.data(), s.size());
    return s.size();
}

ta3c_opt* ta3c_load(const void* buf, uint64_t len) {
    if (!buf) {
        fail("ta3c_load: null buffer");
        return nullptr;
    }
    std::string err;
    Cma* c = Cma::load(std::string(static_cast<char const*>(buf), size_t(len)), &err);
    if (!c) {
        fail(err.c_str());
        return nullptr;
    }
    auto* o = new ta3c_opt;
    o->cma.reset(c);
    return o;
}

const char* ta3c_last_error(void) { return g_err.c_str(); }

int ta3c_sym_eig(uint32_t n, const double* a, double* w, double* v) {
    if (!a || !w || n == 0) return fail("ta3c_sym_eig: bad arguments");
    Mat m(int(n), 0.0);
    std::memcpy(m.a.data(), a, size_t(n) * n * sizeof(double));
    vec ev;
    Mat vv;
    bool const ok = sym_eig(m, ev, v ? &vv : nullptr);
    std::memcpy(w, ev.data(), n * sizeof(double));
    if (v) std::memcpy(v, vv.a.data(), size_t(n) * n * sizeof(double));
    return ok ? 0 : 1;
}

int ta3c_run_test_problem(int kind, int problem, uint32_t dim, uint32_t pop, uint32_t gens, double sigma0,
                          uint32_t seed, double ftol, double xtol, double* champion_f, double* champion_x) {
    if (dim < 2 || pop < 5 || problem < 0 || problem > 2) return fail("ta3c_run_test_problem: bad arguments");
    int const n = int(dim);
    Mat const rot = problem == 2 ? rotation(n) : Mat();
    auto fit = [&](double const* x) -> double {
        if (problem == 0) {
            double s = 0.0;
            for (int i = 0; i < n; ++i) s += x[i] * x[i];
            return s;
        }
        if (problem == 1) return ellipsoid(x, n);
        vec r(size_t(n), 0.0);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) r[size_t(i)] += rot(i, j) * x[j];
        return ellipsoid(r.data(), n);
    };
    vec const lb(size_t(n), -5.0), ub(size_t(n), 5.0);
    Population p(int(pop), lb, ub, seed, fit);
    vec const x0 = p.x[p.best_idx()];
    std::unique_ptr<Cma> cma;
    if (kind == TA3C_SEP)
        cma.reset(new SepCma(x0, lb, ub, sigma0, seed));
    else if (kind == TA3C_DD)
        cma.reset(new DdCma(x0, lb, ub, sigma0, seed, true));
    else
        return fail("ta3c_run_test_problem: bad kind");
    evolve(*cma, p, int(gens), ftol, xtol, [&](int lam, double const* xs, double* fs) {
        for (int i = 0; i < lam; ++i) fs[i] = fit(xs + size_t(i) * n);
    });
    if (champion_f) *champion_f = p.champion_f;
    if (champion_x) std::memcpy(champion_x, p.champion_x.data(), size_t(n) * sizeof(double));
    return 0;
}

} // extern "C"
