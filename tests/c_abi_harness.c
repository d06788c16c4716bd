/* Plain C (C99) caller of librpa_b200: the header compiles as C and the host-only entry points
 * link and run from C, as a Fortran iso_c_binding caller would use them.  Built and run by
 * tests/test_abi.py.  Argument "nogpu": the machine has no GPU, so rpa_b200_create must return
 * RPA_ERR_NO_DEVICE; otherwise a handle is created on device 0 and destroyed. */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "rpa_b200.h"

#define CHECK(cond)                                              \
  do {                                                           \
    if (!(cond)) {                                               \
      fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #cond); \
      return 1;                                                  \
    }                                                            \
  } while (0)

int main(int argc, char** argv) {
  int st;
  int64_t k;
  /* status strings: every code has its own text */
  for (st = RPA_OK; st <= RPA_ERR_INTERNAL; ++st) CHECK(strcmp(rpa_b200_status_string(st), "unknown status") != 0);

  /* frequency grid of a small system (2 occupied, 3 virtual; Fortran order: occupied first) */
  {
    const double e[5] = {-0.9, -0.5, 0.1, 0.4, 1.3};
    double x[64], w[64];
    int64_t n = 0;
    st = rpa_b200_freq_grid(2, 3, e, -3.0, 1e-6, 1e-3, 0, x, w, &n);
    CHECK(st == RPA_OK && n >= 8 && n <= 64);
    for (k = 0; k < n; ++k) CHECK(x[k] > 0.0 && w[k] > 0.0 && (k == 0 || x[k] > x[k - 1]));
    /* a bad gap is reported, not a NaN grid */
    {
      const double bad[5] = {-0.9, 0.5, 0.1, 0.4, 1.3};
      CHECK(rpa_b200_freq_grid(2, 3, bad, -3.0, 1e-6, 1e-3, 0, x, w, &n) == RPA_ERR_INVALID_ARG);
    }
  }

  /* two-body interaction energy E(AB) - E(A) - E(B) */
  {
    const double e3[3] = {-1.0, -0.4, -0.5};
    double eint = 0.0;
    CHECK(rpa_b200_mbe_energy(2, e3, &eint) == RPA_OK && fabs(eint + 0.1) < 1e-15);
    CHECK(rpa_b200_mbe_energy(5, e3, &eint) == RPA_ERR_INVALID_ARG);
  }

  /* handles */
  {
    rpa_b200_handle* h = NULL;
    CHECK(rpa_b200_destroy(NULL) == RPA_OK);
    CHECK(rpa_b200_set_autotune(NULL, 1) == RPA_ERR_INVALID_ARG);
    st = rpa_b200_create(&h, 0, 0);
    if (argc > 1 && strcmp(argv[1], "nogpu") == 0) {
      CHECK(st == RPA_ERR_NO_DEVICE && h == NULL);
    } else {
      CHECK(st == RPA_OK && h != NULL);
      CHECK(rpa_b200_destroy(h) == RPA_OK);
    }
  }
  printf("ok\n");
  return 0;
}
