// What the learned surrogate needs of a simulation: its slot arrays and
// constants, and a way to hand the simulation back a fluid state it did not
// compute itself.
#pragma once

#include "uph_internal.cuh"

struct uph_sim;

namespace uph {

struct SimView {
  DevParams P;
  SlotArrays S;   // current storage buffers (they swap at every re-sort and
                  // every step whose rate pass applies the leapfrog)
  WallTable W;
  cudaStream_t stream;
  unsigned *err;
  int itime;      // steps completed
  bool walls_move;
  int64_t serial;  // distinct for every simulation the process creates
};

SimView sim_view(uph_sim *s);
// The fluid state in the slots now belongs to `nsteps` steps later: advance
// the step counters, put the moving walls at the new time and restart the
// leapfrog at the next step (first-step half kick, as after an upload).  The
// storage re-sort falls due at the next plain step.
uph_status sim_jump(uph_sim *s, int nsteps);
// the device error word as a status (synchronises the stream; the word is sticky)
uph_status sim_check(uph_sim *s);
void sim_count_launches(uph_sim *s, int n);

}  // namespace uph
