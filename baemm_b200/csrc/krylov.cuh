// Batched Krylov solvers on the device, one independent Krylov space per
// column of an n x c row-major block (ld = c), FP64 throughout.
//
//   CG     replaces Tensors::ConjugateGradient as used by ApplyMassInverse.hpp:67-147
//          (A = mass matrix, P = lumped-mass inverse): preconditioned CG per
//          real column, zero initial guess, at most max_iter iterations,
//          column k stops when ||r_k|| <= tol ||b_k||.  Convergence lives in
//          device flags, so the iteration needs no host synchronisation
//          (converged columns are frozen; the launches left after the solve
//          finished return at once).
//   GMRES  replaces Tensors::GMRES<..., Side::Left> (FarField.hpp:538, 706, 828):
//          restarted, left-preconditioned, zero initial guess, CGS2 Arnoldi,
//          complex Givens rotations per column; column k is converged when
//          ||P(b - A x)_k|| <= tol ||P b_k||.  `restart` inner iterations per
//          cycle (gmres_max_iter), `cycles` cycles (gmres_max_restarts).
#pragma once
#include <functional>

#include "ops.cuh"

namespace baemm
{

constexpr int kMaxKrylovColumns = 1024;
constexpr int kMaxRestart = 64;

class CgSolver
{
public:
    ~CgSolver();
    // y = M^-1 b on c real columns (b: n x c with ld ldb, y with ld ldy).
    // Returns true when every column converged; *iterations = iterations run.
    bool solve_mass(const MeshDev &m, bool fp64_values, const double *b, int64_t ldb, double *y, int64_t ldy, int c,
                    double tol, int max_iter, cudaStream_t st, int *iterations);
    // The same in two parts: enqueue_mass only enqueues work on `st` (a fixed
    // launch sequence plus a copy of the convergence flags to pinned host
    // memory, so it can be captured in a CUDA graph); finish synchronises `st`
    // and reads the flags.
    void enqueue_mass(const MeshDev &m, bool fp64_values, const double *b, int64_t ldb, double *y, int64_t ldy, int c,
                      double tol, int max_iter, cudaStream_t st);
    bool finish(cudaStream_t st, int *iterations);
    // Device time of the CG iteration's kernels on the mesh's mass matrix:
    // `iterations` iterations on c real columns (right-hand side all ones,
    // no column allowed to converge), each launch bracketed by CUDA events.
    // ms_out: mean ms per launch of {matvec, update, p update}.
    void profile(const MeshDev &m, bool fp64_values, int c, int iterations, cudaStream_t st, double ms_out[3]);
    // Device time per iteration of cg_block_kernel (the path of meshes of up
    // to 16384 vertices) on c real columns, `iterations` iterations, no column
    // allowed to converge; 0 on larger meshes.
    double profile_block(const MeshDev &m, bool fp64_values, int c, int iterations, cudaStream_t st);

private:
    // partial_: per-block partial sums, group rows and totals of the
    // two-level column sums; counter_: their group and block counters (zero
    // between kernels; zeroed whenever the buffer grows)
    void reserve_totals(int nblk, int S, cudaStream_t st);
    DevBuf<double> x_, r_, z_, p_, q_, col_, partial_;
    DevBuf<int> flags_;
    DevBuf<unsigned int> counter_;
    int *host_flags_ = nullptr;
    bool block_path_ = false;   // the last enqueue_mass ran cg_block_kernel (small meshes)
};

// Device time of one classical Gram-Schmidt pass of a GMRES iteration on an
// n x c complex block against nvec basis vectors (the kernels of the batched
// GMRES below, on scratch blocks of constant values): mean ms per launch of
// {dot products, update}, over `reps` launches each.
void profile_gram_schmidt(int64_t n, int c, int nvec, int reps, cudaStream_t st, double ms_out[2]);

template <class S>   // S = double (real) or double2 (complex)
class GmresSolver
{
public:
    using Op = std::function<void(const S *, S *)>;
    struct Stats { bool converged = false; int iterations = 0; double max_rel_res = 0; };
    ~GmresSolver();
    // x_out = alpha * x + beta * x_out with x the GMRES solution of A x = b.
    Stats solve(int64_t n, int c, int restart, int cycles, const Op &A, const Op &P, S alpha, const S *b,
                int64_t ldb, S beta, S *x_out, int64_t ldx, double tol, cudaStream_t st);
    size_t device_bytes() const;

private:
    DevBuf<S> V_, H_, sn_, g_, h_, y_, w_, tmp_, x_, b_;
    DevBuf<double> cs_, res_, bnorm_, hn_, partial_;
    DevBuf<int> flags_;
    int *host_flags_ = nullptr;
    double *host_res_ = nullptr;
    int host_cap_ = 0;
};

// Helpers with a host result (they synchronise `st`).  `scratch` holds the
// per-block partial sums; it belongs to the caller's context, so it lives on
// the device the stream runs on.
double device_dot(const double *a, const double *b, int64_t n, DevBuf<double> &scratch, cudaStream_t st);
// out_host[k] = ||w[:,k]||_2 for an n x c complex block (ld c)
void device_colnorms(const double2 *w, int64_t n, int c, double *out_host, DevBuf<double> &scratch,
                     cudaStream_t st);

} // namespace baemm
