// Values for the run-time deck of the reference checker build (see deck.cpp).
// Test infrastructure only.
#ifndef OSHUN_REF_DECK_H
#define OSHUN_REF_DECK_H

struct DeckValues {
    int l0, m0, nump, numx_glob, numy_glob;
    double xmin, xmax, ymin, ymax, pmin, pmax;
    double clf_dp, small_dt, t_stop;
    int n_outsteps;
    int NB_algorithms, if_tridiagonal, if_implicit1D;
    double density_np, Zeta;
};

extern DeckValues g_deck;

#endif
