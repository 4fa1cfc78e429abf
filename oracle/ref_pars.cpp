// ORACLE — test infrastructure only.
//
// Definitions of the reference's `Pars` knobs that its FMM sources read
// (global.hpp declares them `extern const`; global.cpp:303-313 and 769-779
// give the shipped values). This translation unit does not include the
// reference's global.hpp, so the objects are writable and the checker can
// choose p, the leaf caps and the root expansion per call. Linked only into
// oracle/_ref/libref2d.so and libref3d.so.
namespace Pars {
int P_max = 10;            // 2D expansion order (global.cpp:311)
double expTree = 1.0;      // root expansion, percent (global.cpp:303)
int par_count_max = 75;    // 2D leaf cap on all particles (global.cpp:312)
int src_count_max = 50;    // 2D leaf cap on sources (global.cpp:313); 3D leaf cap (global.cpp:779)
double xcenter = 0.0;      // domain centre folded into the 3D root box (global.cpp:609-611)
double ycenter = 0.0;
double zcenter = 0.0;
}

extern "C" void refpars_set(int p_max, double exp_tree, int par_max, int src_max) {
    Pars::P_max = p_max;
    Pars::expTree = exp_tree;
    Pars::par_count_max = par_max;
    Pars::src_count_max = src_max;
}
