/*
 * ref_driver.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Host loop appended (by oracle/build.py) after the reference's own kernel
 * sources -- system file, solver file, caller file, concatenated in the order
 * of src/sodeclmgr.cpp:374-503 and compiled as C -- to run them on the CPU.
 * The result, oracle/_ref/libref_<system>_<solver>.so, is the reference's
 * arithmetic executed by gcc, used to validate the oracle restatement and as
 * the timed CPU baseline.  It is never linked into the shipped library.
 *
 * The loop restates src/sodeclmgr.cpp:951-1015: one record of every orbit's
 * state before each launch of `solver_caller`, one after the last launch,
 * layout [record][equation][orbit]; each launch runs the kernel body for
 * every orbit (get_global_id(0) = orbit index), spread over OpenMP threads.
 */
#ifdef _OPENMP
#include <omp.h>
#endif
#include <stddef.h>

int g_sodecl_numeq;
int g_sodecl_numpar;
int g_sodecl_numnoi;
int g_sodecl_numsteps;
long g_sodecl_listsize;
double g_sodecl_dt;
double g_sodecl_eps;
_Thread_local long g_ref_gid;

typedef struct ref_job {
    int neq, npar, nnoi;
    int ksteps;
    double dt;            /* step the program is built with (printed value) */
    long nchunks;         /* launches; records = nchunks + 1 */
    long n;               /* orbits in this job */
    long orbit_offset;    /* global index of the first orbit */
    double *t;            /* [n] in/out */
    double *y;            /* [n][neq] in/out */
    double *p;            /* [n][npar] */
    double *counters;     /* [n] in/out (stochastic build) */
    double *records;      /* [(nchunks+1)][neq][n] or NULL */
    double eps;           /* Newton tolerance (_epsilon1_) */
    int nthreads;
} ref_job;

static void ref_record(const ref_job *job, long c)
{
    if (!job->records) return;
    for (int e = 0; e < job->neq; ++e)
        for (long i = 0; i < job->n; ++i)
            job->records[((size_t)c * job->neq + e) * job->n + i] = job->y[i * job->neq + e];
}

int ref_run(const ref_job *job)
{
    g_sodecl_numeq = job->neq;
    g_sodecl_numpar = job->npar;
    g_sodecl_numnoi = job->nnoi;
    g_sodecl_numsteps = job->ksteps;
    g_sodecl_listsize = job->n;
    g_sodecl_dt = job->dt;
    g_sodecl_eps = job->eps;
#ifdef _OPENMP
    if (job->nthreads > 0) omp_set_num_threads(job->nthreads);
#endif
    /* the kernel indexes its buffers by the global orbit id; shift the base
     * pointers so a job may cover any contiguous range of orbits */
    const long off = job->orbit_offset;
    double *t = job->t - off;
    double *y = job->y - off * job->neq;
    double *p = job->p - off * job->npar;
#ifdef REF_STOCHASTIC
    double *cnt = job->counters - off;
#endif
    for (long c = 0; c < job->nchunks; ++c) {
        ref_record(job, c);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16)
#endif
        for (long i = 0; i < job->n; ++i) {
            g_ref_gid = off + i;
#ifdef REF_STOCHASTIC
            solver_caller(t, y, p, cnt);
#else
            solver_caller(t, y, p);
#endif
        }
    }
    ref_record(job, job->nchunks);
    return 0;
}
