// The ghost-cell method's per-step launch arguments (ghost.cu), shared with the step launch
// set in step.cu.
#pragma once
#include "handle.cuh"

namespace pb
{

struct GhostGeo
{
    int res;
    float h;
    f3 mn;
};

struct GhostStep
{
    GhostGeo g;
    float *grid[3];  // the three time levels, by time index mod 3
    int count, nsolid, first_only, n_listen;
    int listen_cell[8];
    const int *cells, *order, *col, *type, *ghost_idx, *nearest, *solid;
    const float *w, *val, *points;
    float *b, *x, *work;
    int *iters;
};

// the arguments of the per-step ghost kernel for the handle's current ghost system
GhostStep ghost_args(Handle &h, int n_listen, const int *listen_cell);
// one step of the ghost-cell method after the FDTD update of step kstep (one block)
void ghost_launch(const GhostStep &a, const StepState *st, int kstep, int nt, cudaStream_t s);

}  // namespace pb
