// Batched GMRES across contexts (exa_batch.cu): the Arnoldi steps of many independent
// solves of one model advance together, one set of launches per step for all of them.
#pragma once

struct ExaCtx;
struct ExaBatcher;

// A batcher with `capacity` job slots on `device`, run by its own host thread and stream.
int exa_batcher_create(int device, int capacity, ExaBatcher** out);
// Finishes the jobs in flight and frees the batcher.
void exa_batcher_destroy(ExaBatcher* b);
// GMRES on context c's current system through the batcher (blocks until done); same
// results as exa_drv_gmres restricted to what batching supports (exa_batchable).
int exa_batcher_gmres(ExaBatcher* b, ExaCtx& c, int* iters, double* relerr);
// out[4] = {batched steps, kernel launches, jobs done, tuned elements per warp of the matvec}
void exa_batcher_stats(ExaBatcher* b, long long* out);
// Block-Jacobi, MGS, no reduced basis or polynomial preconditioner, condensed blocks up to 64.
bool exa_batchable(const ExaCtx& c);
