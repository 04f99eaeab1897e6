// ref_params_harness.cu — runs the reference's own parameter-file routines
// (test infrastructure).  Compiled by oracle/ref_build.sh together with the
// reference's fun.cu (main renamed); supplies main():
//
//   ref_params_harness save <step> <i_offset_history> <l_offset_Vp> <delta>
//       set_parameters + save_parameters -> ./parameters.txt (fun.cu:1984-2202)
//   ref_params_harness load
//       load_parameters(./parameters.txt) and print the fields it sets
//       (fun.cu:2204-2388)
#include REF_SOURCE
#undef main

int main(int argc, char **argv) {
  if (argc < 2) return 1;
  constants para;
  memset(&para, 0, sizeof(para));
  set_parameters(&para);
  if (!strcmp(argv[1], "save")) {
    para.step = atol(argv[2]);
    para.i_offset_history = atoi(argv[3]);
    para.l_offset_Vp = atof(argv[4]);
    para.delta = atof(argv[5]);
    save_parameters(&para, i_tip_target);
    return 0;
  }
  if (!strcmp(argv[1], "load")) {
    load_parameters(&para);
    printf("%ld %d %.17g %.17g %.17g %d %d %d %d %d %d %.17g %.17g %d %.17g %.17g\n", para.step,
           para.i_offset_history_initial, para.l_offset_Vp_initial, para.delta_initial, para.dt,
           para.i_left_end_initial, para.i_left_end, para.NxT, para.NyT, para.NxT_all, para.NyT_all,
           para.length_sample, para.dtT, para.ratio_dt_dtT, para.Tcold, para.Thot);
    return 0;
  }
  return 1;
}
