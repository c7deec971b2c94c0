/*
 * Drives the gfortran-mangled drop-ins hk_psi_c16_ and ditsp_c16_ of
 * libcpwb200.so the way compiled Fortran calls them: every argument by
 * reference, LOGICAL as a 4-byte int, complex(8) as interleaved doubles, and
 * the lnewanl flag in read-only memory, where gfortran puts a literal such as
 * the .TRUE. that Src/ALFA/berry_derivative.f90:229 passes to hk_psi_c16. A
 * library that stored to lnewanl would die here with SIGSEGV.
 *
 * Usage: dropin_harness DIR. DIR holds dims.txt ("m nb ng nanl mtxds neig
 * mxdsml mxdbnd" then kmscr(1:7)) and the raw input arrays written by
 * tests/test_gpu_dropin_harness.py; the harness writes hpsi1.bin (first call,
 * lnewanl .TRUE.), hpsi2.bin (second call, lnewanl .FALSE., anlga changed in
 * place), ei.bin and ditsp.txt ("ifail neig") from ditsp_c16_.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <unistd.h>

void hk_psi_c16_(const int* mtxd, const int* neig, const double* psi, double* hpsi, int* lnewanl, const int* ng,
                 const int* kgv, const double* ekpg, const int* isort, const double* vscr, const int* kmscr,
                 const double* anlga, const double* xnlkb, const int* nanl, const int* mxddim, const int* mxdbnd,
                 const int* mxdanl, const int* mxdgve, const int* mxdscr);
void ditsp_c16_(const int* ipr, int* ifail, const int* icmax, const int* iguess, const double* epspsi, int* lnewanl,
                int* neig, const int* mtxd, const int* mtxds, double* psi, double* hpsi, double* ei,
                const double* ekpg, const int* isort, const double* vscr, const int* kmscr, const int* ng,
                const int* kgv, const double* anlga, const double* xnlkb, const int* nanl, const double* hamsm,
                const double* hdiag, const int* mxddim, const int* mxdsml, const int* mxdbnd, const int* mxdgve,
                const int* mxdscr, const int* mxdanl);

static const char* g_dir;

static void* load(const char* name, size_t bytes) {
  char path[4096];
  snprintf(path, sizeof path, "%s/%s", g_dir, name);
  FILE* f = fopen(path, "rb");
  if (!f) {
    fprintf(stderr, "cannot open %s\n", path);
    exit(2);
  }
  void* p = calloc(bytes ? bytes : 1, 1);
  if (bytes && fread(p, 1, bytes, f) != bytes) {
    fprintf(stderr, "short read %s\n", path);
    exit(2);
  }
  fclose(f);
  return p;
}

static void save(const char* name, const void* p, size_t bytes) {
  char path[4096];
  snprintf(path, sizeof path, "%s/%s", g_dir, name);
  FILE* f = fopen(path, "wb");
  if (!f || fwrite(p, 1, bytes, f) != bytes) {
    fprintf(stderr, "cannot write %s\n", path);
    exit(2);
  }
  fclose(f);
}

/* a LOGICAL in a page that is mapped read-only before the library sees it */
static int* readonly_logical(int value) {
  const long pg = sysconf(_SC_PAGESIZE);
  int* p = (int*)mmap(NULL, (size_t)pg, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
  if (p == MAP_FAILED) {
    perror("mmap");
    exit(2);
  }
  *p = value;
  if (mprotect(p, (size_t)pg, PROT_READ) != 0) {
    perror("mprotect");
    exit(2);
  }
  return p;
}

int main(int argc, char** argv) {
  if (argc != 2) {
    fprintf(stderr, "usage: %s DIR\n", argv[0]);
    return 2;
  }
  g_dir = argv[1];
  int m, nb, ng, nanl, mtxds, neig, mxdsml, mxdbnd, kmscr[7];
  {
    char path[4096];
    snprintf(path, sizeof path, "%s/dims.txt", g_dir);
    FILE* f = fopen(path, "r");
    if (!f || fscanf(f, "%d %d %d %d %d %d %d %d", &m, &nb, &ng, &nanl, &mtxds, &neig, &mxdsml, &mxdbnd) != 8) {
      fprintf(stderr, "bad dims.txt\n");
      return 2;
    }
    for (int i = 0; i < 7; ++i)
      if (fscanf(f, "%d", &kmscr[i]) != 1) {
        fprintf(stderr, "bad kmscr\n");
        return 2;
      }
    fclose(f);
  }
  const int nv = kmscr[6] * kmscr[4] * kmscr[5];
  int* kgv = (int*)load("kgv.bin", sizeof(int) * 3 * (size_t)ng);
  int* isort = (int*)load("isort.bin", sizeof(int) * (size_t)m);
  double* ekpg = (double*)load("ekpg.bin", sizeof(double) * (size_t)m);
  double* vscr = (double*)load("vscr.bin", sizeof(double) * (size_t)nv);
  double* anl = (double*)load("anl1.bin", 16 * (size_t)m * nanl);
  double* anl2 = (double*)load("anl2.bin", 16 * (size_t)m * nanl);
  double* xnl = (double*)load("xnl.bin", sizeof(double) * (size_t)nanl);
  double* psi = (double*)load("psi.bin", 16 * (size_t)m * nb);
  double* hamsm = (double*)load("hamsm.bin", 16 * (size_t)mxdsml * mxdsml);
  double* hdiag = (double*)load("hdiag.bin", sizeof(double) * (size_t)m);
  double* hpsi = (double*)calloc(2 * (size_t)m * nb, sizeof(double));
  int* lnew_true = readonly_logical(1);
  int* lnew_false = readonly_logical(0);

  /* two H|psi> calls: projectors announced by lnewanl, then changed in place with lnewanl .FALSE. */
  hk_psi_c16_(&m, &nb, psi, hpsi, lnew_true, &ng, kgv, ekpg, isort, vscr, kmscr, anl, xnl, &nanl, &m, &nb, &nanl, &ng,
              &nv);
  save("hpsi1.bin", hpsi, 16 * (size_t)m * nb);
  memcpy(anl, anl2, 16 * (size_t)m * nanl);
  hk_psi_c16_(&m, &nb, psi, hpsi, lnew_false, &ng, kgv, ekpg, isort, vscr, kmscr, anl, xnl, &nanl, &m, &nb, &nanl,
              &ng, &nv);
  save("hpsi2.bin", hpsi, 16 * (size_t)m * nb);

  /* the eigensolver with the changed projectors, lnewanl .TRUE. in read-only memory */
  const int ipr = 0, icmax = 60, iguess = 0;
  const double epspsi = 1e-5;
  int ifail = -1, ne = neig;
  double* P = (double*)calloc(2 * (size_t)m * mxdbnd, sizeof(double));
  double* HP = (double*)calloc(2 * (size_t)m * mxdbnd, sizeof(double));
  double* ei = (double*)calloc((size_t)mxdbnd, sizeof(double));
  ditsp_c16_(&ipr, &ifail, &icmax, &iguess, &epspsi, lnew_true, &ne, &m, &mtxds, P, HP, ei, ekpg, isort, vscr, kmscr,
             &ng, kgv, anl, xnl, &nanl, hamsm, hdiag, &m, &mxdsml, &mxdbnd, &ng, &nv, &nanl);
  save("ei.bin", ei, sizeof(double) * (size_t)ne);
  {
    char path[4096];
    snprintf(path, sizeof path, "%s/ditsp.txt", g_dir);
    FILE* f = fopen(path, "w");
    fprintf(f, "%d %d\n", ifail, ne);
    fclose(f);
  }
  printf("harness ok: lnewanl flags %d %d\n", *lnew_true, *lnew_false);
  return 0;
}
