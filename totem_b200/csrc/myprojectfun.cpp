// myProjectfun with the reference's exact C++ signature (waveCuda.h:10-21), forwarding to the
// engine's C ABI.  Built four times, once per MEX flavour of the reference (mex_cuda.m:19-37):
//   TOTEM_SHIM_PARAM        0 = Peng / Peng-extended rows (waveCudaPengAndCorr*), 1 = Lobato
//   TOTEM_SHIM_TRANSMISSION 0 = STEM (return_result, mid_ceng_mat),
//                           1 = transmission only (potentialx / potentialy), the *P libraries
// The unchanged reference MEX shim waveCuda.cpp links against one of them.  beginRow / beginCol
// arrive already 0-based (waveCuda.cpp:99).  The reference reports nothing on failure; this shim
// writes the engine's status and message to stderr and leaves the outputs untouched.
#include <cstdio>

#include "../../include/totem_b200.h"

#ifndef TOTEM_SHIM_PARAM
#define TOTEM_SHIM_PARAM 0
#endif
#ifndef TOTEM_SHIM_TRANSMISSION
#define TOTEM_SHIM_TRANSMISSION 0
#endif

__attribute__((visibility("default")))
void myProjectfun(double* my_real_w, double* my_imag_w, double* aper, double* atom_slice, double* absorp_n,
                  double* atom_slice_i, double* absorp_n_i, double* proj_coff_mat, double* proj_coff_mat_i,
                  double* kx, double* ky, double* s_2, double* my_real_const, double* my_img_const, double* gfsf,
                  int Height, int Width, int Depth, int P_Height, int P_Width, int Slices, int step, int beginRow,
                  int beginCol, int width_red, double sigma, int w_num, int aper_num, double parameter,
                  double* AperTrue, int* mid_ceng, int ceng_len, double* aper2, double* series_n_corr,
                  double* series_n_i_corr, double* ele_n_corr, double* ele_n_i_corr, double* corr_info_matrix,
                  int cim_len, double* return_result, double* mid_ceng_mat, double* potentialx,
                  double* potentialy) {
  TotemStemArgs a = {};
  a.struct_size = (int)sizeof(TotemStemArgs);
  a.param = TOTEM_SHIM_PARAM ? TOTEM_PARAM_LOBATO : TOTEM_PARAM_PENG;
  a.probe_re = my_real_w;
  a.probe_im = my_imag_w;
  a.aper = aper;
  a.atom_slice = atom_slice;
  a.absorp_n = absorp_n;
  a.atom_slice_i = atom_slice_i;
  a.absorp_n_i = absorp_n_i;
  a.proj_coff_mat = proj_coff_mat;
  a.proj_coff_mat_i = proj_coff_mat_i;
  a.kx = kx;
  a.ky = ky;
  a.s_2 = s_2;
  a.prop_re = my_real_const;
  a.prop_im = my_img_const;
  a.gfsf = gfsf;
  a.height = Height;
  a.width = Width;
  a.depth = Depth;
  a.p_height = P_Height;
  a.p_width = P_Width;
  a.slices = Slices;
  a.step = step;
  a.begin_row = beginRow;
  a.begin_col = beginCol;
  a.width_red = width_red;
  a.sigma = sigma;
  a.w_num = w_num;
  a.aper_num = aper_num;
  a.parameter = parameter;
  a.aper_true = AperTrue;
  a.mid_layer = mid_ceng;
  a.layer_len = ceng_len;
  a.aper2 = aper2;
  a.series_n_corr = series_n_corr;
  a.series_n_i_corr = series_n_i_corr;
  a.ele_n_corr = ele_n_corr;
  a.ele_n_i_corr = ele_n_i_corr;
  a.corr_info_matrix = corr_info_matrix;
  a.cim_len = cim_len;
  TotemStemOut o = {};
  int rc;
#if TOTEM_SHIM_TRANSMISSION
  o.potential_re = potentialx;
  o.potential_im = potentialy;
  rc = totem_transmission_run(&a, &o);
#else
  o.result = return_result;
  o.mid_layer_mat = mid_ceng_mat;
  rc = totem_stem_run(&a, nullptr, &o);
#endif
  if (rc != TOTEM_OK) std::fprintf(stderr, "totem_b200: %s: %s\n", totem_status_string(rc), totem_last_error());
}
