/*
 * ref_driver.c -- harness around the reference's own C PPE solver
 * (src/src_c/mod_poisson_solver.c, decomp_2d.c, mod_fft.c compiled unmodified
 * against shim/mpi.h and shim/fftw3.h).  TEST INFRASTRUCTURE ONLY: it is the
 * checker and the CPU baseline, never the product.
 *
 * It reproduces the caller side of the reference:
 *   - decomp_2d_init(nx,ny,nz,p_row,p_col,{T,T,F})  as mod_mpi.f90:64-69 does
 *     for bctype ('PP','PP','NN');
 *   - neighbor_xyz(6,3) as mod_mpi.f90:87-104 computes it with MPI_CART_SHIFT;
 *   - init_poisson_solver(nx,ny,nz,dx,dy,dzf_global,"PP","PP","NN",neighbor_xyz)
 *     as main.f90:80;  execute_poisson_solver(p) as main.f90:177 on the local
 *     x-pencil block with one ghost layer (mod_variables.f90:39);
 *     free_poisson_solver() as main.f90:273.
 *
 * Two entry points:
 *   ref_ppe_solve(...)  library call (one rank, p_row = p_col = 1);
 *   main()              executable: ref_ppe_run p_row p_col nx ny nz dx dy
 *                       dzf.bin in.bin out.bin [nrep]; forks p_row*p_col
 *                       ranks when > 1 (needed for PDD with p_col partitions).
 * Arrays are the global ghosted (nx+2)(ny+2)(nz+2) FP64 field in Fortran
 * order; only the interior is read and written, like the reference.
 */
#define _GNU_SOURCE
#include <mpi.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <time.h>

#include "decomp_2d.h"

extern void init_poisson_solver(int nx_global, int ny_global, int nz_global, double dx, double dy,
                                double *dzf_global, char bctype_x[], char bctype_y[], char bctype_z[],
                                int neighbor_xyz[3][6]);
extern void execute_poisson_solver(double *var);
extern void free_poisson_solver(void);

static double now_s(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* neighbour table of mod_mpi.f90:87-104; C [pencil][dir], dir = W,E,S,N,B,T */
static void make_neighbors(int nb[3][6])
{
    nb[0][0] = MPI_PROC_NULL;
    nb[0][1] = MPI_PROC_NULL;
    MPI_Cart_shift(decomp_2d_comm_cart_x, 0, 1, &nb[0][2], &nb[0][3]);
    MPI_Cart_shift(decomp_2d_comm_cart_x, 1, 1, &nb[0][4], &nb[0][5]);
    MPI_Cart_shift(decomp_2d_comm_cart_y, 0, 1, &nb[1][0], &nb[1][1]);
    nb[1][2] = MPI_PROC_NULL;
    nb[1][3] = MPI_PROC_NULL;
    MPI_Cart_shift(decomp_2d_comm_cart_y, 1, 1, &nb[1][4], &nb[1][5]);
    MPI_Cart_shift(decomp_2d_comm_cart_z, 0, 1, &nb[2][0], &nb[2][1]);
    MPI_Cart_shift(decomp_2d_comm_cart_z, 1, 1, &nb[2][2], &nb[2][3]);
    nb[2][4] = MPI_PROC_NULL;
    nb[2][5] = MPI_PROC_NULL;
}

typedef struct {
    int p_row, p_col, nx, ny, nz;
    double dx, dy;
    double *dzf;     /* nz+2 */
    const double *in; /* global ghosted */
    double *out;     /* global ghosted (shared when ranks are forked) */
    int nrep;
    double t_init, t_exec; /* rank 0 timings */
    double *timing;  /* shared [2] */
} run_args;

static int rank_main(int rank, void *vp)
{
    run_args *a = (run_args *)vp;
    bool periodic[3] = {true, true, false};
    decomp_2d_init(a->nx, a->ny, a->nz, a->p_row, a->p_col, periodic);
    int nb[3][6];
    make_neighbors(nb);
    const int *st = decomp_main.xst, *sz = decomp_main.xsz;
    const size_t gx = (size_t)a->nx + 2, gy = (size_t)a->ny + 2;
    const size_t lx = (size_t)sz[0] + 2, ly = (size_t)sz[1] + 2, lz = (size_t)sz[2] + 2;
    double *var = (double *)calloc(lx * ly * lz, sizeof(double));
    for (int k = 1; k <= sz[2]; k++)
        for (int j = 1; j <= sz[1]; j++)
            memcpy(&var[(size_t)1 + lx * ((size_t)j + ly * (size_t)k)],
                   &a->in[(size_t)st[0] + gx * ((size_t)(st[1] - 1 + j) + gy * (size_t)(st[2] - 1 + k))],
                   sizeof(double) * (size_t)sz[0]);
    char bx[] = "PP", by[] = "PP", bz[] = "NN";
    double t0 = now_s();
    init_poisson_solver(a->nx, a->ny, a->nz, a->dx, a->dy, a->dzf, bx, by, bz, nb);
    double t1 = now_s();
    /* the first call produces the result; further calls only time the solve
       on a fresh copy of the same input */
    double *work = NULL;
    if (a->nrep > 1) {
        work = (double *)malloc(sizeof(double) * lx * ly * lz);
        memcpy(work, var, sizeof(double) * lx * ly * lz);
    }
    execute_poisson_solver(var);
    double t2 = now_s();
    double texec = t2 - t1;
    if (a->nrep > 1) {
        MPI_Barrier(MPI_COMM_WORLD);
        double t3 = now_s();
        for (int r = 1; r < a->nrep; r++) execute_poisson_solver(work);
        MPI_Barrier(MPI_COMM_WORLD);
        texec = (now_s() - t3) / (double)(a->nrep - 1);
        free(work);
    }
    for (int k = 1; k <= sz[2]; k++)
        for (int j = 1; j <= sz[1]; j++)
            memcpy(&a->out[(size_t)st[0] + gx * ((size_t)(st[1] - 1 + j) + gy * (size_t)(st[2] - 1 + k))],
                   &var[(size_t)1 + lx * ((size_t)j + ly * (size_t)k)], sizeof(double) * (size_t)sz[0]);
    free_poisson_solver();
    decomp_2d_finalize();
    free(var);
    if (rank == 0 && a->timing) {
        a->timing[0] = t1 - t0;
        a->timing[1] = texec;
    }
    return 0;
}

/* Library entry: one rank.  in/out may alias. */
int ref_ppe_solve(int nx, int ny, int nz, double dx, double dy, const double *dzf_global, const double *in,
                  double *out)
{
    size_t n = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    double *dzf = (double *)malloc(sizeof(double) * (size_t)(nz + 2));
    memcpy(dzf, dzf_global, sizeof(double) * (size_t)(nz + 2));
    double *inc = (double *)malloc(sizeof(double) * n);
    memcpy(inc, in, sizeof(double) * n);
    if (out != in) memcpy(out, in, sizeof(double) * n);
    double timing[2];
    run_args a = {1, 1, nx, ny, nz, dx, dy, dzf, inc, out, 1, 0, 0, timing};
    int rc = oracle_mpi_run(1, 0, rank_main, &a);
    free(inc);
    free(dzf);
    return rc;
}


/* Persistent one-rank instance (init once, execute many times), as the
 * reference driver uses it (main.f90:80,177,273).  Used for timing. */
static double *g_dzf_keep = NULL;
int ref_ppe_setup(int nx, int ny, int nz, double dx, double dy, const double *dzf_global)
{
    bool periodic[3] = {true, true, false};
    decomp_2d_init(nx, ny, nz, 1, 1, periodic);
    int nb[3][6];
    make_neighbors(nb);
    g_dzf_keep = (double *)malloc(sizeof(double) * (size_t)(nz + 2));
    memcpy(g_dzf_keep, dzf_global, sizeof(double) * (size_t)(nz + 2));
    char bx[] = "PP", by[] = "PP", bz[] = "NN";
    init_poisson_solver(nx, ny, nz, dx, dy, g_dzf_keep, bx, by, bz, nb);
    return 0;
}

void ref_ppe_exec(double *var) { execute_poisson_solver(var); }

void ref_ppe_teardown(void)
{
    free_poisson_solver();
    decomp_2d_finalize();
    free(g_dzf_keep);
    g_dzf_keep = NULL;
}

static int read_file(const char *path, void *buf, size_t bytes)
{
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    size_t r = fread(buf, 1, bytes, f);
    fclose(f);
    return r == bytes ? 0 : -1;
}

#ifndef REF_DRIVER_NO_MAIN
int main(int argc, char **argv)
{
    if (argc < 11) {
        fprintf(stderr, "usage: %s p_row p_col nx ny nz dx dy dzf.bin in.bin out.bin [nrep]\n", argv[0]);
        return 2;
    }
    run_args a;
    memset(&a, 0, sizeof(a));
    a.p_row = atoi(argv[1]);
    a.p_col = atoi(argv[2]);
    a.nx = atoi(argv[3]);
    a.ny = atoi(argv[4]);
    a.nz = atoi(argv[5]);
    a.dx = strtod(argv[6], NULL);
    a.dy = strtod(argv[7], NULL);
    a.nrep = argc > 11 ? atoi(argv[11]) : 1;
    size_t n = (size_t)(a.nx + 2) * (a.ny + 2) * (a.nz + 2);
    a.dzf = (double *)malloc(sizeof(double) * (size_t)(a.nz + 2));
    double *in = (double *)malloc(sizeof(double) * n);
    if (read_file(argv[8], a.dzf, sizeof(double) * (size_t)(a.nz + 2)) || read_file(argv[9], in, sizeof(double) * n)) {
        fprintf(stderr, "cannot read inputs\n");
        return 2;
    }
    a.in = in;
    a.out = (double *)mmap(NULL, sizeof(double) * n, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    a.timing = (double *)mmap(NULL, 4096, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    memcpy(a.out, in, sizeof(double) * n);
    long msg = (long)sizeof(double) * (long)(a.nx + 2) * (long)(a.ny + 2) * (long)(a.nz + 2);
    int nprocs = a.p_row * a.p_col;
    if (nprocs > 1) msg = 2 * (msg / nprocs) + 4096;
    int rc = oracle_mpi_run(nprocs, msg, rank_main, &a);
    if (rc != 0) {
        fprintf(stderr, "reference run failed (%d)\n", rc);
        return 1;
    }
    FILE *f = fopen(argv[10], "wb");
    if (!f || fwrite(a.out, sizeof(double), n, f) != n) {
        fprintf(stderr, "cannot write output\n");
        return 1;
    }
    fclose(f);
    printf("init_s %.6e exec_s %.6e\n", a.timing[0], a.timing[1]);
    return 0;
}
#endif
