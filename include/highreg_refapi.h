// highreg_refapi.h — C++ drop-in layer with the reference's own call
// signatures (libhighreg_refapi.so, built over the C ABI of highreg_b200.h).
//
// A program written against the reference's two-surface evaluators
// (highreg_stokes_2surf: KITC.h:99-118, stokeslets.h:9-29, stresslets.h:9-30)
// links against this library instead of KITC.cpp, stokeslets.cpp and
// stresslets.cpp and runs its boundary sums on the B200. The point and target
// records must be layout-identical to the reference's (2S/utilities.h:30-53),
// because the caller allocates them; they are declared here with the same
// member names, types and order.
//
// Treecode parameters are run-time here (the reference fixes them at compile
// time in KITC.h:14-17; defaults P = 6, N0 = 1000, theta = 0.6), as are the
// surface centres used for the treecode root box (defaults: the reference's
// ctr1 / ctr2, 2S/utilities.h:19-26).
#ifndef HIGHREG_REFAPI_H
#define HIGHREG_REFAPI_H

#include <vector>

struct Surf_point {
  Surf_point() : x(3, 0), f(3, 0), g(3, 0), Nrml(3, 0), Area(0), plane(0), left(0), right(0), up(0), down(0) {}
  std::vector<double> x;
  std::vector<double> f;
  std::vector<double> g;
  std::vector<double> Nrml;
  double Area;
  int plane, left, right, up, down;
};

struct Target_point {
  Target_point()
      : x(0), y(0), z(0), nrst_x(0), nrst_y(0), nrst_z(0), nrst_Nrml(3, 0), nrst_f(3, 0), nrst_g(3, 0),
        u(0), v(0), w(0), nrst(0), i1(0), i2(0), i3(0), b(0) {}
  double x, y, z;
  double nrst_x, nrst_y, nrst_z;
  std::vector<double> nrst_Nrml, nrst_f, nrst_g;
  double u, v, w;
  int nrst;
  int i1;
  int i2;
  int i3;
  double b;
};

// Treecode evaluators (2S/KITC.h:99-118)
void eval_Stokes_SL_onSurf_tree(int surf_num, double h, double DEL, int N_quad,
                                const std::vector<Surf_point>& Surfc, int N_target,
                                const std::vector<Target_point>& Target, std::vector<double>& SL);
void eval_Stokes_SL_offSurf_tree(int surf_num, double h, double DEL, int N_quad,
                                 const std::vector<Surf_point>& Surfc, int N_target,
                                 const std::vector<Target_point>& Target, std::vector<double>& SL);
void eval_Stokes_DL_onSurf_tree(int surf_num, double h, double DEL, int N_quad,
                                const std::vector<Surf_point>& Surfc, int N_target,
                                const std::vector<Target_point>& Target, std::vector<double>& DL);
void eval_Stokes_DL_offSurf_tree(int surf_num, double h, double DEL, int N_quad,
                                 const std::vector<Surf_point>& Surfc, int N_target,
                                 const std::vector<Target_point>& Target, std::vector<double>& SL);

// Direct evaluators (2S/stokeslets.h:9-29, 2S/stresslets.h:9-30)
void eval_Stokes_SL_offSurf(double h, double DEL, int N_quad, const std::vector<Surf_point>& Surfc,
                            int N_target, const std::vector<Target_point>& Target,
                            std::vector<double>& SL);
void eval_Stokes_SL_onSurf(double DEL, int N_quad, const std::vector<Surf_point>& Surfc, int N_target,
                           const std::vector<Target_point>& Target, std::vector<double>& SL_vec);
void eval_Stokes_DL_offSurf(double h, double DEL, int N_quad, const std::vector<Surf_point>& Surfc,
                            int N_target, std::vector<Target_point>& Target,
                            std::vector<double>& DL_vec);
void eval_Stokes_DL_onSurf(double DEL, int N_quad, const std::vector<Surf_point>& Surfc, int N_target,
                           std::vector<Target_point>& Target, std::vector<double>& DL_vec);

// Run-time settings of this layer (no counterpart in the reference).
extern "C" void hr_refapi_set_tree(int P, int N0, double theta);
extern "C" void hr_refapi_set_center(int surf_num, double x, double y, double z);
extern "C" void hr_refapi_set_device(int device);

#endif
