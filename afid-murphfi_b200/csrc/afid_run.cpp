// afid_run — command-line drop-in for the reference's `afid` executable on the flow +
// temperature path: reads bou.in from the working directory (ReadInputFile.F90:20) and runs
// the main loop (main.F90:281-422) with the substep on the GPU.
//   afid_run [--steps N] [--seed S] [--mixed] [--stats K] [--outputdir D] [bou.in]
// With --outputdir the run reads D/continua_*.h5 when NREAD = 1 and writes the SAVE_3D frames and
// the final continua files there, as the reference does in outputdir/.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "afid_continua.h"
#include "afid_host.h"

static void on_step(int ntime, double time, double dt, double nu, double ke, void *) {
  std::printf("  T = %.4e NTIME = %9d DT = %.4e  Nu_vol = %.6f  KE = %.6e\n", time, ntime, dt, nu, ke);
}

int main(int argc, char **argv) {
  const char *path = "bou.in";
  const char *dir = nullptr;
  int steps = -1, stats = 0, prec = AFID_PREC_FP64;
  unsigned long long seed = 20261203ULL;
  for (int a = 1; a < argc; ++a) {
    if (!std::strcmp(argv[a], "--steps") && a + 1 < argc) steps = std::atoi(argv[++a]);
    else if (!std::strcmp(argv[a], "--seed") && a + 1 < argc) seed = std::strtoull(argv[++a], nullptr, 10);
    else if (!std::strcmp(argv[a], "--stats") && a + 1 < argc) stats = std::atoi(argv[++a]);
    else if (!std::strcmp(argv[a], "--mixed")) prec = AFID_PREC_MIXED;
    else if (!std::strcmp(argv[a], "--outputdir") && a + 1 < argc) dir = argv[++a];
    else path = argv[a];
  }
  afid_input_t in;
  int s = afid_read_bou_in(path, &in);
  if (s != AFID_OK) {
    std::fprintf(stderr, "afid_run: cannot read %s: %s\n", path, afid_gpu_status_string(s));
    return 2;
  }
  afid_run_stats_t st;
  s = afid_run_io(&in, prec, seed, steps, stats, stats > 0 ? on_step : nullptr, nullptr, dir, &st);
  if (s != AFID_OK) {
    std::fprintf(stderr, "afid_run: %s\n", afid_gpu_status_string(s));
    return 1;
  }
  const double cells = (double)in.nxm * in.nym * in.nzm;
  std::printf("steps %d  time %.6e  dt %.4e  errorcode %d  maxdiv %.3e  Nu_vol %.6f  KE %.6e\n", st.steps_done,
              st.time, st.dt, st.errorcode, st.divmax, st.nu_vol, st.ke);
  std::printf("Mcell-RK3-steps/s %.2f  (%.3f s)\n", cells * st.steps_done / st.seconds / 1e6, st.seconds);
  return (st.errorcode == 0 || st.errorcode == 333 || st.errorcode == 555) ? 0 : 3;
}
