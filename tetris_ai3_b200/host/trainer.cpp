// Island CMA-ES trainer (include/ta3b_trainer.h): the reference's Trainer2
// (ta3_trainer/src/trainer2.cpp) over pagmo's archipelago, restated as a
// lock-step loop that scores every island's generation in one evaluator call.
#include "../../include/ta3b_trainer.h"

#include "../../include/ta3b.h"
#include "../../include/ta3b_cma.h"
#include "../../include/ta3b_surrogate.h"
#include "cmaes.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <memory>
#include <numeric>
#include <random>
#include <string>
#include <thread>
#include <vector>

using namespace ta3b::host;

namespace {

thread_local std::string g_create_err;

using clock_t_ = std::chrono::steady_clock;
double seconds_since(clock_t_::time_point t0) {
    return std::chrono::duration<double>(clock_t_::now() - t0).count();
}

// xoshiro256** seeded through splitmix64 (ta3_sim/incl/ta3/sim/utility/xoshiro256ss.hpp:20-48),
// the trainer's _generator (trainer2.hpp:91)
struct Xoshiro {
    uint64_t s[4];
    explicit Xoshiro(uint64_t seed) {
        for (auto& v : s) {
            seed += 0x9e3779b97f4a7c15ULL;
            uint64_t z = seed;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
            v = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t operator()() {
        uint64_t const r = rotl(s[1] * 5, 7) * 9;
        uint64_t const t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
};

// fn(i) for i in [0, n) on up to n host threads (the islands' optimisers are
// independent, so the result does not depend on the interleaving)
template<class F>
void for_islands(uint32_t n, F const& fn) {
    if (n <= 1) {
        for (uint32_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(n - 1);
    for (uint32_t i = 1; i < n; ++i) th.emplace_back([&fn, i] { fn(i); });
    fn(0);
    for (auto& t : th) t.join();
}

// Spearman rank correlation (average ranks for ties)
std::vector<double> ranks(std::vector<double> const& v) {
    size_t const n = v.size();
    std::vector<size_t> o(n);
    std::iota(o.begin(), o.end(), size_t{0});
    std::sort(o.begin(), o.end(), [&](size_t a, size_t b) { return v[a] < v[b]; });
    std::vector<double> r(n);
    for (size_t i = 0; i < n;) {
        size_t j = i;
        while (j + 1 < n && v[o[j + 1]] == v[o[i]]) ++j;
        double const avg = 0.5 * double(i + j);
        for (size_t k = i; k <= j; ++k) r[o[k]] = avg;
        i = j + 1;
    }
    return r;
}

double spearman(std::vector<double> const& a, std::vector<double> const& b) {
    size_t const n = a.size();
    if (n < 3) return 0.0 / 0.0;
    std::vector<double> const ra = ranks(a), rb = ranks(b);
    double ma = 0, mb = 0;
    for (size_t i = 0; i < n; ++i) {
        ma += ra[i];
        mb += rb[i];
    }
    ma /= double(n);
    mb /= double(n);
    double sab = 0, saa = 0, sbb = 0;
    for (size_t i = 0; i < n; ++i) {
        sab += (ra[i] - ma) * (rb[i] - mb);
        saa += (ra[i] - ma) * (ra[i] - ma);
        sbb += (rb[i] - mb) * (rb[i] - mb);
    }
    if (saa == 0 || sbb == 0) return 0.0;
    return sab / std::sqrt(saa * sbb);
}

// the built-in surrogate: the GPU MLP behind include/ta3b_surrogate.h, 97 -> 128 ->
// 128 -> 2 for v11's parameter vectors, num_params -> 256 -> 256 -> 2 for any other size
constexpr uint32_t kV11Params = 97, kWideSurrogateHidden = 256;
struct GpuSurrogate {
    ta3s_model* model = nullptr;
    ta3w_model* wide = nullptr;
    uint32_t epochs = 40, batch = 256, trainings = 0;
    float lr = 1e-3f, weight_decay = 0.0f;      // plain Adam (the kernels also take a decoupled decay)
    ~GpuSurrogate() {
        if (model) ta3s_destroy(model);
        if (wide) ta3w_destroy(wide);
    }
};

int gpu_sur_train(void* user, const float* x, const float* y, uint32_t n, uint32_t) {
    auto* s = static_cast<GpuSurrogate*>(user);
    float loss = 0.f;
    uint32_t const seed = 0x5A11u + s->trainings++;
    if (s->wide)
        return ta3w_set_data(s->wide, x, y, n) ||
               ta3w_train(s->wide, s->epochs, s->batch, s->lr, s->weight_decay, seed, &loss);
    if (ta3s_set_data(s->model, x, y, n)) return 1;
    return ta3s_train(s->model, s->epochs, s->batch, s->lr, s->weight_decay, seed, &loss);
}

int gpu_sur_predict(void* user, const float* x, uint32_t n, uint32_t, float* mean_out) {
    auto* s = static_cast<GpuSurrogate*>(user);
    return s->wide ? ta3w_predict(s->wide, x, n, mean_out, nullptr) : ta3s_predict(s->model, x, n, mean_out, nullptr);
}

// the built-in score function: the GPU evaluator behind include/ta3b.h
int gpu_score(void* user, const float* weights, uint32_t num_models, uint32_t num_params, const uint64_t* seeds,
              uint32_t num_games, uint32_t max_moves, float* score_out, uint32_t* pieces_out) {
    return ta3b_eval(static_cast<ta3b_ctx*>(user), weights, num_models, num_params, seeds, num_games, max_moves,
                     score_out, pieces_out, nullptr);
}

struct Island {
    std::unique_ptr<Cma> cma;
    std::vector<vec> x;          // the island population (last fully evaluated candidates)
    vec f;
    vec champion_x;
    double champion_f = 0.0 / 0.0;
    bool has_migrant = false;    // the archipelago's migrant database entry (select_best, rate 1)
    vec migrant_x;
    double migrant_f = 0.0;

    void set_xf(size_t i, double const* xi, double fi) {
        x[i].assign(xi, xi + x[i].size());
        f[i] = fi;
        if (champion_x.empty() || less_f(fi, champion_f)) {
            champion_x.assign(xi, xi + x[i].size());
            champion_f = fi;
        }
    }
    size_t best() const { return size_t(std::min_element(f.begin(), f.end(), less_f) - f.begin()); }
    size_t worst() const { return size_t(std::max_element(f.begin(), f.end(), less_f) - f.begin()); }
};

} // namespace

// One island group's evaluator: islands i with i % groups == g are scored by group g's
// score function, on its own host thread (the built-in one: its own GPU context).
struct Group {
    ta3t_score_fn fn = nullptr;
    void* user = nullptr;
    ta3b_ctx* gpu = nullptr;          // owned (built-in evaluator)
};

struct ta3t_trainer {
    ta3t_config cfg{};
    std::vector<Group> groups;
    std::unique_ptr<GpuSurrogate> gpu_sur;
    bool has_surrogate = false;
    ta3t_surrogate sur{};
    Xoshiro generator{0};
    std::mt19937 select_rng;         // surrogate's random extra picks (separate from the seed stream)
    uint64_t game_seed = 0;          // _iterationSeed (trainer2.hpp:100), 0 until the first cycle
    std::vector<Island> islands;
    std::vector<double> lb, ub;
    ta3t_stats st{};
    std::string err;
    // surrogate archive: every fully evaluated candidate (x as float) and its mean score
    std::vector<float> arch_x;
    std::vector<float> arch_y;
    std::vector<uint64_t> arch_gen;
    bool sur_active = false;

    ~ta3t_trainer() {
        for (auto& g : groups)
            if (g.gpu) ta3b_destroy(g.gpu);
    }

    int fail(std::string m) {
        err = std::move(m);
        return 1;
    }

    // Score n candidates (row-major doubles, island-major: n / islands rows per island):
    // fitness = -mean score. One evaluator call per island group, the groups concurrently.
    int score(size_t n, double const* xs, double* fitness, float* mean_out) {
        uint32_t const P = cfg.num_params, G = cfg.games, I = cfg.islands;
        std::vector<float> w(n * P);
        for (size_t i = 0; i < n * P; ++i) w[i] = static_cast<float>(xs[i]);   // tetris_problem2.cpp:35-38
        std::vector<uint64_t> seeds(G);
        ta3b_simulate_seeds(game_seed, G, seeds.data());
        std::vector<float> sc(n * G);
        std::vector<uint32_t> pc(n * G);
        auto const t0 = clock_t_::now();
        size_t const D = groups.size();
        std::vector<int> rcs(D, 0);
        if (D == 1) {
            rcs[0] = groups[0].fn(groups[0].user, w.data(), uint32_t(n), P, seeds.data(), G, cfg.max_moves, sc.data(),
                                  pc.data());
        } else {
            // island group g: islands g, g + D, ...; its rows gathered, scored, scattered back
            size_t const rows = n / I;
            auto run = [&](size_t g) {
                std::vector<uint32_t> isl;
                for (uint32_t i = uint32_t(g); i < I; i += uint32_t(D)) isl.push_back(i);
                size_t const m = isl.size() * rows;
                if (m == 0) return;
                std::vector<float> wg(m * P), sg(m * G);
                std::vector<uint32_t> pg(m * G);
                for (size_t k = 0; k < isl.size(); ++k)
                    std::memcpy(&wg[k * rows * P], &w[isl[k] * rows * P], rows * P * sizeof(float));
                rcs[g] = groups[g].fn(groups[g].user, wg.data(), uint32_t(m), P, seeds.data(), G, cfg.max_moves,
                                      sg.data(), pg.data());
                for (size_t k = 0; k < isl.size(); ++k) {
                    std::memcpy(&sc[isl[k] * rows * G], &sg[k * rows * G], rows * G * sizeof(float));
                    std::memcpy(&pc[isl[k] * rows * G], &pg[k * rows * G], rows * G * sizeof(uint32_t));
                }
            };
            std::vector<std::thread> th;
            for (size_t g = 1; g < D; ++g) th.emplace_back(run, g);
            run(0);
            for (auto& t : th) t.join();
        }
        st.eval_seconds += seconds_since(t0);
        for (size_t g = 0; g < D; ++g)
            if (rcs[g])
                return fail(groups[g].gpu ? std::string("evaluator: ") + ta3b_last_error(groups[g].gpu)
                                          : "score function failed (island group " + std::to_string(g) + ")");
        for (size_t m = 0; m < n; ++m) {
            double sum = 0.0;                                            // tetris_problem2.cpp:59-64
            for (uint32_t g = 0; g < G; ++g) sum += double(sc[m * G + g]);
            double const mean = sum / double(G);
            fitness[m] = -mean;
            if (mean_out) mean_out[m] = float(mean);
            for (uint32_t g = 0; g < G; ++g) st.pieces += pc[m * G + g];
        }
        st.sims += n * G;
        st.evaluations += n;
        return 0;
    }

    ta3t_surrogate sur_builtin{};

    // fns / users: one score function per island group (a NULL entry: the built-in GPU evaluator
    // on device cfg.device + group)
    int init(ta3t_config const* c, uint32_t num_groups, ta3t_score_fn const* fns, void* const* users,
             ta3t_surrogate const* s, std::string const* state) {
        cfg = *c;
        if (num_groups == 0 || num_groups > 64) return fail("ta3t_create: 1 to 64 island groups");
        if (cfg.islands == 0 || cfg.population < 5 || cfg.games == 0 || cfg.num_params == 0 ||
            cfg.gens_per_iteration == 0 || cfg.iterations_per_cycle == 0)
            return fail("ta3t_create: islands, games, num_params, gens and iterations must be positive, population >= 5");
        if (!(cfg.sigma0 > 0.0) || !(cfg.upper > cfg.lower)) return fail("ta3t_create: bad sigma0 or bounds");
        if (cfg.algo != TA3C_SEP && cfg.algo != TA3C_DD) return fail("ta3t_create: algo must be TA3C_SEP or TA3C_DD");
        if (cfg.surrogate_start_gen && !s) {
            gpu_sur = std::make_unique<GpuSurrogate>();
            if (cfg.num_params == kV11Params) {
                gpu_sur->model = ta3s_create(c->device, uint32_t(cfg.training_seed));
                if (!gpu_sur->model) return fail(std::string("surrogate: ") + ta3s_last_error(nullptr));
            } else {
                gpu_sur->wide = ta3w_create(c->device, cfg.num_params, kWideSurrogateHidden, uint32_t(cfg.training_seed));
                if (!gpu_sur->wide) return fail(std::string("surrogate: ") + ta3w_last_error(nullptr));
            }
            if (cfg.surrogate_epochs) gpu_sur->epochs = cfg.surrogate_epochs;
            if (cfg.surrogate_batch) gpu_sur->batch = cfg.surrogate_batch;
            if (cfg.surrogate_lr > 0) gpu_sur->lr = float(cfg.surrogate_lr);
            sur_builtin = ta3t_surrogate{gpu_sur.get(), gpu_sur_train, gpu_sur_predict};
            s = &sur_builtin;
        }
        if (cfg.surrogate_start_gen) {
            if (!s || !s->train || !s->predict) return fail("ta3t_create: pre-screening needs a surrogate");
            if (cfg.surrogate_top + cfg.surrogate_random < 5 ||
                cfg.surrogate_top + cfg.surrogate_random > cfg.surrogate_sample || cfg.surrogate_retrain == 0)
                return fail("ta3t_create: need 5 <= top + random <= sample and retrain > 0");
        }
        if (s) {
            has_surrogate = true;
            sur = *s;
        }
        groups.resize(num_groups);
        for (uint32_t g = 0; g < num_groups; ++g) {
            if (fns && fns[g]) {
                groups[g].fn = fns[g];
                groups[g].user = users ? users[g] : nullptr;
            } else {
                ta3b_config const gc{c->device + int(g), 0, 0};
                groups[g].gpu = ta3b_create(&gc);
                if (!groups[g].gpu) return fail(std::string("evaluator: ") + ta3b_last_error(nullptr));
                groups[g].fn = gpu_score;
                groups[g].user = groups[g].gpu;
            }
        }
        st.last_rho = 0.0 / 0.0;
        generator = Xoshiro(cfg.training_seed);
        select_rng.seed(uint32_t(cfg.training_seed ^ (cfg.training_seed >> 32)) ^ 0x5u);
        uint32_t const P = cfg.num_params;
        lb.assign(P, cfg.lower);
        ub.assign(P, cfg.upper);

        // trainer2.cpp:144-168: archipelago seed, per-island population seeds, then optimiser seeds
        std::mt19937 arch_eng(static_cast<unsigned>(generator()));
        std::uniform_int_distribution<unsigned> udist;
        islands.resize(cfg.islands);
        uint32_t const N = cfg.population;
        std::vector<double> xs(size_t(cfg.islands) * N * P);
        for (uint32_t i = 0; i < cfg.islands; ++i) {
            std::mt19937 eng(udist(arch_eng));
            for (uint32_t k = 0; k < N; ++k)
                for (uint32_t j = 0; j < P; ++j)
                    xs[(size_t(i) * N + k) * P + j] = std::uniform_real_distribution<double>(lb[j], ub[j])(eng);
        }
        // initial populations: one evaluator call, game seed 0 (trainer2.cpp:45-49 before the first cycle)
        std::vector<double> fit(size_t(cfg.islands) * N);
        std::vector<float> means(fit.size());
        auto const t0 = clock_t_::now();
        if (score(fit.size(), xs.data(), fit.data(), means.data())) return 1;
        for (uint32_t i = 0; i < cfg.islands; ++i) {
            Island& is = islands[i];
            is.x.assign(N, vec(P));
            is.f.assign(N, 0.0);
            for (uint32_t k = 0; k < N; ++k) is.set_xf(k, &xs[(size_t(i) * N + k) * P], fit[size_t(i) * N + k]);
            if (state) {
                std::string e;
                is.cma.reset(Cma::load(*state, &e));
                if (!is.cma) return fail("ta3t_create_from_state: " + e);
                if (is.cma->dim() != int(P)) return fail("ta3t_create_from_state: saved dimension differs");
            } else if (cfg.algo == TA3C_SEP) {
                is.cma.reset(new SepCma(is.x[is.best()], lb, ub, cfg.sigma0, 0));
            } else {
                is.cma.reset(new DdCma(is.x[is.best()], lb, ub, cfg.sigma0, 0, true));
            }
        }
        archive(xs.data(), means.data(), fit.size(), 0);
        for (auto& is : islands) is.cma->reseed(static_cast<unsigned>(generator()));
        st.host_seconds += seconds_since(t0) - st.eval_seconds;
        st.best_fitness = best_fitness();
        return 0;
    }

    void archive(double const* xs, float const* means, size_t n, uint64_t gen) {
        if (!has_surrogate) return;
        size_t const P = cfg.num_params;
        size_t const base = arch_x.size();
        arch_x.resize(base + n * P);
        for (size_t i = 0; i < n * P; ++i) arch_x[base + i] = float(xs[i]);
        arch_y.insert(arch_y.end(), means, means + n);
        arch_gen.insert(arch_gen.end(), n, gen);
    }

    double best_fitness() const {
        // trainer2.cpp:295-303
        double best = std::numeric_limits<double>::max();
        for (auto const& is : islands)
            if (!is.champion_x.empty() && is.champion_f < best) best = is.champion_f;
        return best;
    }

    // retrain on everything but the last generation, gate on that held-out slice
    int retrain(uint64_t gen) {
        size_t const P = cfg.num_params;
        std::vector<float> tx, ty, hx;
        std::vector<double> hy;
        uint64_t const first = cfg.surrogate_window && gen > uint64_t(cfg.surrogate_window) + 1
                                   ? gen - 1 - cfg.surrogate_window : 0;
        for (size_t i = 0; i < arch_y.size(); ++i) {
            if (arch_gen[i] < first) continue;
            bool const held = arch_gen[i] + 1 == gen;
            float const* xi = &arch_x[i * P];
            if (held) {
                hx.insert(hx.end(), xi, xi + P);
                hy.push_back(arch_y[i]);
            } else {
                tx.insert(tx.end(), xi, xi + P);
                ty.push_back(arch_y[i]);
            }
        }
        if (ty.size() < 16 || hy.size() < 3) {
            sur_active = false;
            return 0;
        }
        auto const t0 = clock_t_::now();
        if (sur.train(sur.user, tx.data(), ty.data(), uint32_t(ty.size()), uint32_t(P)))
            return fail("surrogate training failed");
        std::vector<float> pred(hy.size());
        if (sur.predict(sur.user, hx.data(), uint32_t(hy.size()), uint32_t(P), pred.data()))
            return fail("surrogate prediction failed");
        st.surrogate_seconds += seconds_since(t0);
        st.surrogate_trainings++;
        std::vector<double> pd(pred.begin(), pred.end());
        st.last_rho = spearman(pd, hy);
        sur_active = st.last_rho >= cfg.surrogate_min_rho;
        return 0;
    }

    int generation() {
        auto const t_start = clock_t_::now();
        double const eval0 = st.eval_seconds, sur0 = st.surrogate_seconds;
        uint64_t const gen = st.generation + 1;
        uint32_t const P = cfg.num_params, N = cfg.population, I = cfg.islands;
        bool const screening_period = cfg.surrogate_start_gen && gen >= cfg.surrogate_start_gen;
        if (screening_period && (gen - cfg.surrogate_start_gen) % cfg.surrogate_retrain == 0)
            if (retrain(gen)) return 1;
        bool const pre = screening_period && sur_active;
        uint32_t const n_ask = pre ? cfg.surrogate_sample : N;

        std::vector<double> asked(size_t(I) * n_ask * P);
        for_islands(I, [&](uint32_t i) { islands[i].cma->ask(int(n_ask), &asked[size_t(i) * n_ask * P]); });

        // which candidates get full evaluation
        std::vector<std::vector<int>> chosen(I);
        if (pre) {
            std::vector<float> xf(asked.size());
            for (size_t k = 0; k < asked.size(); ++k) xf[k] = float(asked[k]);
            std::vector<float> pred(size_t(I) * n_ask);
            auto const t0 = clock_t_::now();
            if (sur.predict(sur.user, xf.data(), uint32_t(pred.size()), P, pred.data()))
                return fail("surrogate prediction failed");
            st.surrogate_seconds += seconds_since(t0);
            for (uint32_t i = 0; i < I; ++i) {
                std::vector<int> o(n_ask);
                std::iota(o.begin(), o.end(), 0);
                float const* pi = &pred[size_t(i) * n_ask];
                // highest predicted mean score first; index breaks ties
                std::stable_sort(o.begin(), o.end(), [pi](int a, int b) { return pi[a] > pi[b]; });
                std::vector<int> c(o.begin(), o.begin() + cfg.surrogate_top);
                std::vector<int> rest(o.begin() + cfg.surrogate_top, o.end());
                for (uint32_t r = 0; r < cfg.surrogate_random; ++r) {
                    size_t const j = r + std::uniform_int_distribution<size_t>(0, rest.size() - 1 - r)(select_rng);
                    std::swap(rest[r], rest[j]);
                    c.push_back(rest[r]);
                }
                chosen[i] = std::move(c);
            }
        } else {
            for (uint32_t i = 0; i < I; ++i) {
                chosen[i].resize(n_ask);
                std::iota(chosen[i].begin(), chosen[i].end(), 0);
            }
        }

        size_t total = 0;
        for (auto const& c : chosen) total += c.size();
        std::vector<double> xs(total * P), fit(total);
        std::vector<float> means(total);
        size_t row = 0;
        for (uint32_t i = 0; i < I; ++i)
            for (int c : chosen[i]) {
                std::memcpy(&xs[row * P], &asked[(size_t(i) * n_ask + size_t(c)) * P], P * sizeof(double));
                ++row;
            }
        if (score(total, xs.data(), fit.data(), means.data())) return 1;

        std::vector<size_t> first_row(I + 1, 0);
        for (uint32_t i = 0; i < I; ++i) first_row[i + 1] = first_row[i] + chosen[i].size();
        for_islands(I, [&](uint32_t i) {
            Island& is = islands[i];
            size_t const k = chosen[i].size(), r0 = first_row[i];
            is.x.assign(k, vec(P));
            is.f.assign(k, 0.0);
            for (size_t j = 0; j < k; ++j) is.set_xf(j, &xs[(r0 + j) * P], fit[r0 + j]);
            is.cma->tell(int(k), chosen[i].data(), &fit[r0]);
        });
        if (pre) {
            std::vector<float> xf(total * P);
            for (size_t k = 0; k < xf.size(); ++k) xf[k] = float(xs[k]);
            std::vector<float> pred(total);
            auto const t0 = clock_t_::now();
            if (sur.predict(sur.user, xf.data(), uint32_t(total), P, pred.data()))
                return fail("surrogate prediction failed");
            st.surrogate_seconds += seconds_since(t0);
            std::vector<double> pd(pred.begin(), pred.end()), md(means.begin(), means.end());
            st.last_rho = spearman(pd, md);
        }
        archive(xs.data(), means.data(), total, gen);
        st.generation = gen;
        st.best_fitness = best_fitness();
        st.surrogate_active = pre ? 1u : 0u;
        st.host_seconds += seconds_since(t_start) - (st.eval_seconds - eval0) - (st.surrogate_seconds - sur0);
        return 0;
    }

    // ring{1} migration (trainer2.cpp:145-146): each island pulls the best individual
    // of one randomly chosen ring neighbour (edge weight 1) and, if it is better,
    // it replaces the island's worst (select_best / fair_replace, rate 1)
    void migrate() {
        size_t const I = islands.size();
        if (I < 2) return;
        for (size_t i = 0; i < I; ++i) {
            size_t const prev = (i + I - 1) % I, next = (i + 1) % I;
            size_t const from = (I == 2 || std::uniform_int_distribution<int>(0, 1)(select_rng) == 0) ? prev : next;
            Island const& src = islands[from];
            Island& dst = islands[i];
            if (!src.has_migrant) continue;
            size_t const w = dst.worst();
            if (less_f(src.migrant_f, dst.f[w])) dst.set_xf(w, src.migrant_x.data(), src.migrant_f);
        }
    }

    void publish_migrants() {
        for (auto& is : islands) {
            size_t const b = is.best();
            is.migrant_x = is.x[b];
            is.migrant_f = is.f[b];
            is.has_migrant = true;
        }
    }

    int iteration() {
        migrate();
        for (auto& is : islands) is.cma->new_evolve();
        for (uint32_t g = 0; g < cfg.gens_per_iteration; ++g)
            if (generation()) return 1;
        publish_migrants();
        st.iteration++;
        return 0;
    }

    void next_game_seed() {
        game_seed = generator();
        st.game_seed = game_seed;
    }
};

extern "C" {

void ta3t_default_config(ta3t_config* c) {
    if (!c) return;
    *c = ta3t_config{};
    c->islands = 4;
    c->population = 50;
    c->gens_per_iteration = 10;
    c->iterations_per_cycle = 10;
    c->games = 30;
    c->max_moves = 300;
    c->algo = TA3C_DD;
    c->num_params = TA3B_NUM_PARAMS;
    c->training_seed = 0x3e28df7b1811145bULL;
    c->sigma0 = 1.3;
    c->lower = -2.0;
    c->upper = 2.0;
    c->device = 0;
    c->surrogate_start_gen = 0;
    c->surrogate_sample = 200;
    c->surrogate_top = 50;
    c->surrogate_random = 5;
    c->surrogate_retrain = 10;
    c->surrogate_min_rho = 0.6;
    c->surrogate_epochs = 40;
    c->surrogate_batch = 256;
    c->surrogate_lr = 1e-3;
    c->surrogate_window = 0;
    c->num_devices = 1;
}

static ta3t_trainer* create(const ta3t_config* cfg, std::string const* state, uint32_t groups,
                            ta3t_score_fn const* fns, void* const* users, const ta3t_surrogate* s) {
    if (!cfg) {
        g_create_err = "ta3t_create: null config";
        return nullptr;
    }
    auto* t = new ta3t_trainer;
    if (t->init(cfg, groups, fns, users, s, state)) {
        g_create_err = t->err;
        delete t;
        return nullptr;
    }
    return t;
}

ta3t_trainer* ta3t_create(const ta3t_config* cfg, ta3t_score_fn score_fn, void* user, const ta3t_surrogate* s) {
    // the built-in evaluator: one island group per device (cfg->num_devices, at least one)
    uint32_t const groups = score_fn || !cfg || cfg->num_devices < 2 ? 1u : cfg->num_devices;
    std::vector<ta3t_score_fn> fns(groups, score_fn);
    std::vector<void*> users(groups, user);
    return create(cfg, nullptr, groups, fns.data(), users.data(), s);
}

ta3t_trainer* ta3t_create_groups(const ta3t_config* cfg, uint32_t num_groups, const ta3t_score_fn* score_fns,
                                 void* const* users, const ta3t_surrogate* s) {
    if (num_groups == 0 || !score_fns) {
        g_create_err = "ta3t_create_groups: need at least one score function";
        return nullptr;
    }
    for (uint32_t g = 0; g < num_groups; ++g)
        if (!score_fns[g]) {
            g_create_err = "ta3t_create_groups: null score function";
            return nullptr;
        }
    return create(cfg, nullptr, num_groups, score_fns, users, s);
}

ta3t_trainer* ta3t_create_from_state(const ta3t_config* cfg, const char* state_path, ta3t_score_fn score_fn,
                                     void* user, const ta3t_surrogate* s) {
    std::ifstream f(state_path ? state_path : "", std::ios::binary);
    if (!f) {
        g_create_err = "ta3t_create_from_state: cannot open the state file";
        return nullptr;
    }
    std::string const blob((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    uint32_t const groups = score_fn || !cfg || cfg->num_devices < 2 ? 1u : cfg->num_devices;
    std::vector<ta3t_score_fn> fns(groups, score_fn);
    std::vector<void*> users(groups, user);
    return create(cfg, &blob, groups, fns.data(), users.data(), s);
}

void ta3t_destroy(ta3t_trainer* t) { delete t; }

const char* ta3t_last_error(const ta3t_trainer* t) { return t ? t->err.c_str() : g_create_err.c_str(); }

int ta3t_next_game_seed(ta3t_trainer* t) {
    if (!t) return 1;
    t->next_game_seed();
    return 0;
}

int ta3t_run_generation(ta3t_trainer* t) { return t ? t->generation() : 1; }

int ta3t_run_iteration(ta3t_trainer* t) { return t ? t->iteration() : 1; }

int ta3t_run(ta3t_trainer* t, uint32_t iterations) {
    if (!t) return 1;
    for (uint32_t k = 0; k < iterations; ++k) {
        if (t->st.iteration % t->cfg.iterations_per_cycle == 0) t->next_game_seed();   // trainer2.cpp:379-381
        if (t->iteration()) return 1;
    }
    return 0;
}

int ta3t_get_stats(const ta3t_trainer* t, ta3t_stats* out) {
    if (!t || !out) return 1;
    *out = t->st;
    out->surrogate_active = t->sur_active ? 1u : 0u;
    return 0;
}

int ta3t_champion(const ta3t_trainer* t, uint32_t island, double* x_out, double* f_out) {
    if (!t || island >= t->islands.size()) return 1;
    auto const& is = t->islands[island];
    if (x_out) std::memcpy(x_out, is.champion_x.data(), is.champion_x.size() * sizeof(double));
    if (f_out) *f_out = is.champion_f;
    return 0;
}

int ta3t_island_whiten(const ta3t_trainer* t, uint32_t island, const double* x, uint32_t n, double* z_out) {
    if (!t || island >= t->islands.size() || (n && (!x || !z_out))) return 1;
    t->islands[island].cma->whiten(int(n), x, z_out);
    return 0;
}

int ta3t_island_mean(const ta3t_trainer* t, uint32_t island, double* x_out) {
    if (!t || island >= t->islands.size() || !x_out) return 1;
    auto const& m = t->islands[island].cma->mean();
    std::memcpy(x_out, m.data(), m.size() * sizeof(double));
    return 0;
}

int ta3t_write_champ(const char* path, const double* x, uint64_t n) {
    std::ofstream f(path ? path : "", std::ios::binary | std::ios::trunc);
    if (!f || (n && !x)) return 1;
    f.write(reinterpret_cast<char const*>(&n), sizeof n);
    f.write(reinterpret_cast<char const*>(x), std::streamsize(n * sizeof(double)));
    return f ? 0 : 1;
}

uint64_t ta3t_read_champ(const char* path, double* x_out, uint64_t cap) {
    std::ifstream f(path ? path : "", std::ios::binary | std::ios::ate);
    if (!f) return 0;
    auto const size = uint64_t(f.tellg());
    f.seekg(0);
    uint64_t n = 0;
    if (!f.read(reinterpret_cast<char*>(&n), sizeof n)) return 0;
    if (size < sizeof n || n != (size - sizeof n) / sizeof(double)) return 0;   // count must match the file
    std::vector<double> v(n);
    if (!f.read(reinterpret_cast<char*>(v.data()), std::streamsize(n * sizeof(double)))) return 0;
    if (x_out) std::memcpy(x_out, v.data(), std::min(n, cap) * sizeof(double));
    return n;
}

int ta3t_save_state(const ta3t_trainer* t, const char* state_path) {
    if (!t || !state_path) return 1;
    // trainer2.cpp:217-224: the best island (lowest champion fitness)
    size_t best = 0;
    double bf = std::numeric_limits<double>::max();
    for (size_t i = 0; i < t->islands.size(); ++i)
        if (!t->islands[i].champion_x.empty() && t->islands[i].champion_f < bf) {
            bf = t->islands[i].champion_f;
            best = i;
        }
    std::string const blob = t->islands[best].cma->save();
    {
        std::ofstream f(state_path, std::ios::binary | std::ios::trunc);
        if (!f) return 1;
        f.write(blob.data(), std::streamsize(blob.size()));
        if (!f) return 1;
    }
    std::string champ = state_path;
    size_t const dot = champ.find_last_of('.');
    size_t const slash = champ.find_last_of('/');
    if (dot != std::string::npos && (slash == std::string::npos || dot > slash)) champ.resize(dot);
    champ += ".champ";
    auto const& cx = t->islands[best].champion_x;
    return ta3t_write_champ(champ.c_str(), cx.data(), cx.size());
}

} // extern "C"
