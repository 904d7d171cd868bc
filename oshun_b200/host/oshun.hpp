// C++ host layer over the C ABI (include/oshun_b200.h) with the shapes of the
// reference's hot-path classes, so the reference's main loop
// (OSHUN-1/main.cpp:40-134) can call the B200 path with its own call order:
//
//   reference                               this header
//   Stat (decl-state.h:302)                 oshun_b200::State
//   Explicit_Method / Runge_Kutta_4         oshun_b200::Runge_Kutta_4
//     (decl-RK.h:24-80, def-RK.cpp:49-153)
//   Actions::Adv (def-Actions.cpp:73-94)    oshun_b200::Actions::Adv
//   Explicit_EC_FP::loop                    oshun_b200::Explicit_EC_FP::loop
//     (def-FokkerPlanck.cpp:590-625)
//   Euler_Backward::advance_1 / advance_lm  oshun_b200::Euler_Backward
//     (def-FokkerPlanck.cpp:1270-1304)
//
// The state lives on the GPU for the whole run; State::upload/download move
// it in the reference's storage order (complex128, harmonics ind(l,m), p
// fastest, no guard cells).  Errors become oshun_b200::Error exceptions
// carrying the oshun_status code (the C ABI itself never throws).
#pragma once

#include <complex>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "oshun_b200.h"

namespace oshun_b200 {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& what)
        : std::runtime_error(what + ": " + oshun_last_error()), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

inline void check(int rc, const char* what) {
    if (rc != OSHUN_OK) throw Error(rc, what);
}

inline std::size_t num_harmonics(int l0, int m0) {
    return static_cast<std::size_t>(((m0 + 1) * (2 * l0 - m0 + 2)) / 2);
}

// ind(l,m) of OSHUN-1/def-State.cpp:420-427
inline int harmonic_index(int l, int m, int m0) {
    return (l < m0 + 1) ? (l * (l + 1)) / 2 + m : l * (m0 + 1) - (m0 * (m0 + 1)) / 2 + m;
}

// The device-resident state of one run (replaces Stat).
class State {
public:
    explicit State(const oshun_cfg& cfg) : cfg_(cfg) { check(oshun_create(&cfg, &h_), "oshun_create"); }
    ~State() { if (h_) oshun_destroy(h_); }
    State(const State&) = delete;
    State& operator=(const State&) = delete;

    const oshun_cfg& cfg() const { return cfg_; }
    oshun_handle handle() const { return h_; }
    std::size_t harmonic_elems() const {
        return num_harmonics(cfg_.l0, cfg_.m0) * static_cast<std::size_t>(cfg_.numy) * cfg_.numx * cfg_.nump;
    }
    std::size_t field_elems() const { return 6u * static_cast<std::size_t>(cfg_.numy) * cfg_.numx; }

    void upload(const std::vector<std::complex<double>>& f, const std::vector<std::complex<double>>& fields) {
        if (f.size() != harmonic_elems() || fields.size() != field_elems())
            throw std::invalid_argument("State::upload: wrong sizes");
        check(oshun_upload(h_, reinterpret_cast<const double*>(f.data()),
                           reinterpret_cast<const double*>(fields.data())), "oshun_upload");
    }
    void download(std::vector<std::complex<double>>& f, std::vector<std::complex<double>>& fields) const {
        f.resize(harmonic_elems());
        fields.resize(field_elems());
        check(oshun_download(h_, reinterpret_cast<double*>(f.data()), reinterpret_cast<double*>(fields.data())),
              "oshun_download");
    }
    void synchronize() const { check(oshun_synchronize(h_), "oshun_synchronize"); }

private:
    oshun_cfg cfg_;
    oshun_handle h_ = nullptr;
};

// Actions (def-Actions.cpp:57-94): the slope of the current state.
class Actions {
public:
    explicit Actions(State& Y) : Y_(Y) {}
    // slope = F(Y) in the storage order of State::download
    void Adv(std::vector<std::complex<double>>& slope_f, std::vector<std::complex<double>>& slope_fields) {
        slope_f.resize(Y_.harmonic_elems());
        slope_fields.resize(Y_.field_elems());
        check(oshun_rhs(Y_.handle(), reinterpret_cast<double*>(slope_f.data()),
                        reinterpret_cast<double*>(slope_fields.data())), "oshun_rhs");
    }

private:
    State& Y_;
};

// Runge_Kutta_4 with the Explicit_Method interface (decl-RK.h:24-36).
class Runge_Kutta_4 {
public:
    // tout_start: the output step the clock starts at; dt_out as in the deck
    Runge_Kutta_4(State& Y, int tout_start, double dt_out)
        : Y_(Y), dt_out_(dt_out), tout_(static_cast<double>(tout_start) * dt_out + dt_out) {
        // num_h = int(dt_out/CLF)+1, h = dt_out/num_h (def-RK.cpp:60-61) is the
        // caller's cfg.dt; keep num_h for the main loop
        num_h_ = static_cast<std::size_t>(dt_out / Y.cfg().dt + 0.5);
        if (num_h_ == 0) num_h_ = 1;
    }
    Runge_Kutta_4& advance_p1() { check(oshun_rk4_step(Y_.handle()), "oshun_rk4_step"); return *this; }
    Runge_Kutta_4& advance_p2() { return *this; }   // no-op for explicit E (def-RK.cpp:149)
    double& tout() { return tout_; }
    double time() const {
        double t = 0.0;
        check(oshun_time(Y_.handle(), &t), "oshun_time");
        return t;
    }
    std::size_t numh() const { return num_h_; }

private:
    State& Y_;
    double dt_out_;
    double tout_;
    std::size_t num_h_ = 1;
};

// Explicit_EC_FP (decl-fokkerplanck.h:140-149): f00 e-e collisions.
class Explicit_EC_FP {
public:
    explicit Explicit_EC_FP(State& Y) : Y_(Y) {}
    void loop(const double& tnew) { check(oshun_collide_ee(Y_.handle(), tnew), "oshun_collide_ee"); }

private:
    State& Y_;
};

// Euler_Backward (decl-fokkerplanck.h:289-299): implicit f_lm collisions.
class Euler_Backward {
public:
    explicit Euler_Backward(State& Y) : Y_(Y) {}
    void advance_1(const double& tnew) { check(oshun_collide_f1(Y_.handle(), tnew), "oshun_collide_f1"); }
    void advance_lm(const double& tnew) { check(oshun_collide_flm(Y_.handle(), tnew), "oshun_collide_flm"); }

private:
    State& Y_;
};

}  // namespace oshun_b200
