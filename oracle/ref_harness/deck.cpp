// Run-time input deck for the reference checker build.
//
// Test infrastructure only: this file is linked with the reference's own
// hot-path sources (OSHUN-1 def-State.cpp, def-VlasovMax.cpp, def-Actions.cpp,
// def-RK.cpp, def-FokkerPlanck.cpp, def-Nmethods.cpp, compiled unmodified
// from the reference tree) to make the CPU checker `oracle/_ref/oshun_ref`.
//
// The reference compiles its deck in (OSHUN-1/def-Input.cpp:64-303, read
// through the singleton OSHUN-1/def-Input.cpp:391-394).  This file provides
// the same symbols (declared in OSHUN-1/decl-input.h:59-205) but takes the
// values from `g_deck`, which the harness fills before the first call of
// Inputdata::IN().  The derived quantities follow the reference's rules:
//   * guard cells: numx = numx_glob + 2*RKLevel (def-Input.cpp:156-158)
//   * axes: Axis(n, min, max) is i*(max-min)/(n-1) + min; the local x and y
//     axes are the global ones shifted left by RKLevel cells
//     (def-Input.cpp:313-327)
//   * dt_out = t_stop / n_outsteps, CLF = clf_dp (def-Input.cpp:320,332-334)
#include <iostream>
#include <vector>
#include <valarray>
#include <complex>
#include <math.h>

#include "matrices.h"
#include "decl-input.h"
#include "deck.h"

DeckValues g_deck;

Inputdata::input_list::input_list() {
    NnodesX = 1; NnodesY = 1;
    l0 = g_deck.l0; m0 = g_deck.m0;
    nump = g_deck.nump; numx_glob = g_deck.numx_glob; numy_glob = g_deck.numy_glob;
    xmin = g_deck.xmin; xmax = g_deck.xmax;
    ymin = g_deck.ymin; ymax = g_deck.ymax;
    pmin = g_deck.pmin; pmax = g_deck.pmax;
    clf_dp = g_deck.clf_dp;
    if_implicitES = false;   // the implicit-E path solves the full electromagnetic case
    if_implicit1D = g_deck.if_implicit1D != 0;
    small_dt = g_deck.small_dt;
    smaller_dt = g_deck.small_dt;
    NB_algorithms = g_deck.NB_algorithms;
    if_tridiagonal = g_deck.if_tridiagonal != 0;
    implicit_E = false;
    RKLevel = 4;
    n_outsteps = g_deck.n_outsteps;
    t_stop = g_deck.t_stop;
    restart_time = 0; n_restarts = 1;
    bndX = 0; bndY = 0;
    lnLambda = 10.0;
    Zeta = g_deck.Zeta;
    density_np = g_deck.density_np;
    numx = numx_glob + 2 * RKLevel;
    numy = numy_glob + 2 * RKLevel;
    // every moment of Parallel_Output::nonrelativistic_moments on, in the
    // reference's normalised units (def-Input.cpp:197-253, 170-172)
    o_Vx = o_Vy = o_VxVx = o_VyVy = o_VzVz = o_VxVy = o_VxVz = o_VyVz = true;
    o_Vsq = o_Qx = o_Qy = o_Pressure = o_Temperature = o_ND = o_Nu = true;
    denormalize_fields = false;
    denormalize_length = false;
}

Inputdata::decl_input::decl_input(input_list in)
    : l0(in.l0), m0(in.m0),
      pr(in.nump, in.pmin, in.pmax),
      x(in.numx, in.xmin, in.xmax),
      xglob(in.numx_glob, in.xmin, in.xmax),
      y(in.numy, in.ymin, in.ymax),
      yglob(in.numy_glob, in.ymin, in.ymax),
      CLF(in.clf_dp) {
    const double dxg = xglob.dx();
    x(0) = xglob(0) - in.RKLevel * dxg;
    for (size_t i = 1; i < x.dim(); ++i) x(i) = x(i - 1) + dxg;
    const double dyg = yglob.dx();
    y(0) = yglob(0) - in.RKLevel * dyg;
    for (size_t i = 1; i < y.dim(); ++i) y(i) = y(i - 1) + dyg;
}

Inputdata::decl_control::decl_control(input_list in)
    : n_out(in.n_outsteps), tstop(in.t_stop) {
    dt_out = tstop / double(n_out);
}

Inputdata::decl_output::decl_output(input_list in)
    : px(4, 1.0f), p1(4, 1.0f), p2(4, 1.0f), p3(4, 1.0f) {}

Inputdata::Input::Input() {
    ilist = new input_list();
    in = new decl_input(*ilist);
    control = new decl_control(*ilist);
    out = new decl_output(*ilist);
}
Inputdata::Input::~Input() {
    delete ilist; delete in; delete control; delete out;
}
Inputdata::input_list& Inputdata::Input::list() const { return *ilist; }
Inputdata::decl_input& Inputdata::Input::inp() const { return *in; }
Inputdata::decl_control& Inputdata::Input::cont() const { return *control; }
Inputdata::decl_output& Inputdata::Input::outp() const { return *out; }

Inputdata::Input& Inputdata::IN() {
    static Inputdata::Input the_input;
    return the_input;
}
