// pb_gmres.cuh — batched preconditioned GMRES over the dense FP64 systems of a batch.
#pragma once
#include <vector>
#include "pb_lu.cuh"

#define PB_GMRES_MAXM 60     // Krylov dimension per cycle (GMRES_MAXIT, iterative.c:29)

struct pb_gmres_args {
    pb_lu_engine *eng;
    int n;                  // order
    int nsys;               // systems (frequencies) of the batch
    int nrhs;               // right-hand sides per system
    const double2 *A;       // FP64 matrices, row-major, stride A_stride
    long A_stride;
    const float2 *lu;       // FP32 LU factors of the anchor frequencies, stride lu_stride
    long lu_stride;
    const int *perm;        // [anchors][n] row permutations of those factors (device)
    const int *lu_of;       // [nsys] anchor of each system (host)
    const double2 *b;       // [nsys][nrhs][n] right-hand sides (device)
    double2 *x;             // [nsys][nrhs][n] solutions (device)
    double eta;             // normwise backward-error target
    int m;                  // Krylov dimension (<= PB_GMRES_MAXM)
    int max_cycles;         // GMRES cycles (the first run plus restarts)
};

struct pb_gmres_result {
    long iters_total;       // Arnoldi steps summed over systems
    int iters_max;
    int solved;
};

// state[s] on entry: 0 = solve, anything else = skip. On return: 1 = converged,
// 2 = not converged (the caller refactorises those), others unchanged.
int pb_gmres_batched(const pb_gmres_args &a, std::vector<int> &state, pb_gmres_result *res);
