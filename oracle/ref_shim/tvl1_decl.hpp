/*
 * Forced-include header (g++ -include) used only when compiling the
 * reference's sequential TV-L1 (src/tvl1/sequential/tvl1.cpp) into
 * oracle/_ref.  It defines the reference header's include guard
 * (DUAL_TVL1_OPTIC_FLOW_H, src/tvl1/sequential/tvl1.hpp:1-2), so tvl1.cpp's own
 * `#include "tvl1.hpp"` is skipped and this declaration is used instead.  The
 * reference source files are compiled where they lie, unmodified.
 *
 * Differences from src/tvl1/sequential/tvl1.hpp, and why:
 *  - MAX_ITERATIONS (tvl1.hpp:6, a constexpr 300) becomes a run-time global so
 *    the harness can set the inner-iteration cap (50 for the 1024x436 workload,
 *    1..k for per-iteration checks).
 *  - Every member is public, so the harness can call dualTVL1() on one pyramid
 *    level and read the dual variables p after it.  All data members stay in
 *    one access section, in the reference's declaration order.
 *  - <cstddef> is included (tvl1.hpp uses size_t without it).
 * The constants PRESMOOTHING_SIGMA and GRAD_IS_ZERO keep the reference values
 * (tvl1.hpp:7-8).
 */
#ifndef DUAL_TVL1_OPTIC_FLOW_H
#define DUAL_TVL1_OPTIC_FLOW_H

#include <cstddef>
#include <cstdint>

extern std::size_t MAX_ITERATIONS;
constexpr float PRESMOOTHING_SIGMA{0.8f};
constexpr float GRAD_IS_ZERO{1E-10};

class TV_L1 {
public:
    TV_L1(int width, int height, float tau = 0.25, float lambda = 0.15,
          float theta = 0.3, int nscales = 100, float zfactor = 0.5, int warps = 5,
          float epsilon = 0.01);
    ~TV_L1();
    float *getU() { return _u; }
    void runDualTVL1Multiscale(uint8_t *I0, uint8_t *I1);

    void dualTVL1(const float *I0, const float *I1, float *u1, float *u2, int nx, int ny);
    void image_normalization(const float *I0, const float *I1, float *I0n, float *I1n, int size);
    void convertToFloat(int size, const uint8_t *I0, const uint8_t *I1, float *_I0, float *_I1);

    float *_u;
    float **_I0s, **_I1s, **_u1s, **_u2s;
    int *_nx, *_ny;
    float *_I1x, *_I1y, *_I1w, *_I1wx, *_I1wy, *_rho_c, *_v1, *_v2, *_p11, *_p12,
        *_p21, *_p22, *_grad, *_div_p1, *_div_p2, *_g1, *_g2;
    int _width;
    int _height;
    float _tau;
    float _lambda;
    float _theta;
    int _nscales;
    float _zfactor;
    int _warps;
    float _epsilon;
};

#endif
