#pragma once
/* Gaussian shells and multi-shell-pairs.
 *
 * The two structs keep the reference's field order and types exactly
 * (skel/simint/shell/shell.h:18-32 and :47-85, built with
 * SIMINT_OSTEI_MAXDER = 1 so alpha2/beta2 are present), because callers
 * (C, C++ and the Fortran bindings of skel/simint/simint.f90:6-40) read and
 * fill them directly.  Primitive-pair arrays use the reference's 8-wide
 * padding: after every SIMINT_NSHELL_SIMD (16) shell pairs the element count
 * is rounded up to a multiple of SIMINT_SIMD_LEN (8), padding entries having
 * alpha = 1, prefac = 0 and screen = 0 (shell.c:538-570). */

#include <stddef.h>
#include "simint/ostei/ostei_config.h"

#define SIMINT_SCREEN_NONE         0
#define SIMINT_SCREEN_SCHWARZ      1
#define SIMINT_SCREEN_FASTSCHWARZ  2

#ifdef __cplusplus
extern "C" {
#endif

struct simint_shell
{
    int am;          /* angular momentum (0 = s) */
    int nprim;       /* number of primitives */
    double x, y, z;  /* centre, bohr */
    double * alpha;  /* exponents [nprim] */
    double * coef;   /* contraction coefficients [nprim] */
    size_t memsize;  /* bytes owned through ptr */
    void * ptr;      /* the one allocation holding alpha and coef */
};

struct simint_multi_shellpair
{
    int am1;            /* AM of the first shell of every pair */
    int am2;            /* AM of the second shell of every pair */
    int nprim;          /* primitive pairs stored, padding excluded */
    int nshell12;       /* shell pairs stored */
    int nshell12_clip;  /* shell pairs to compute (<= nshell12) */
    int * nprim12;      /* primitive pairs per shell pair [nshell12] */
    double * AB_x;      /* A - B per shell pair [nshell12] */
    double * AB_y;
    double * AB_z;
    double * x;         /* Gaussian-product centre P per primitive pair */
    double * y;
    double * z;
    double * PA_x;      /* P - A */
    double * PA_y;
    double * PA_z;
    double * PB_x;      /* P - B */
    double * PB_y;
    double * PB_z;
    double * alpha;     /* a + b */
#if SIMINT_OSTEI_MAXDER > 0
    double * alpha2;    /* 2a (a+b on off-diagonal pairs of a shell with itself) */
    double * beta2;     /* 2b (likewise) */
#endif
    double * prefac;    /* cA cB exp(-ab/(a+b) |AB|^2) sqrt(2 pi^(5/2)) / (a+b) */
    double * screen;    /* per primitive pair screening value, or NULL */
    double screen_max;  /* maximum of screen[] */
    size_t memsize;     /* bytes owned through ptr */
    void * ptr;         /* the one allocation holding every array above */
};

/* Two shells are the same shell when they share storage (shell.h:88-94);
 * a pair of a shell with itself keeps only the i >= j primitive triangle. */
static inline int compare_shell(struct simint_shell const * A,
                                struct simint_shell const * B)
{
    return A->nprim == B->nprim && A->ptr == B->ptr;
}

/* Replaces simint_initialize_shell (shell.h:104, shell.c:188-192). */
void simint_initialize_shell(struct simint_shell * G);
/* Replaces simint_initialize_shells (shell.h:116, shell.c:194-198). */
void simint_initialize_shells(int n, struct simint_shell * G);
/* Replaces simint_allocate_shell (shell.h:125, shell.c:202-214). */
void simint_allocate_shell(int nprim, struct simint_shell * G);
/* Replaces simint_free_shell (shell.h:132, shell.c:217-223). */
void simint_free_shell(struct simint_shell * G);
/* Replaces simint_free_shells (shell.h:142, shell.c:225-229). */
void simint_free_shells(int n, struct simint_shell * G);
/* Replaces simint_copy_shell (shell.h:150-151, shell.c:231-242). */
void simint_copy_shell(struct simint_shell const * src, struct simint_shell * dest);
/* Replaces simint_normalize_shells (shell.h:161, shell.c:248-278). */
void simint_normalize_shells(int n, struct simint_shell * G);
/* Replaces simint_create_shell (shell.h:185-188, shell.c:281-294). */
void simint_create_shell(int nprim, int am, double x, double y, double z,
                         double const * alpha, double const * coef,
                         struct simint_shell * G);
/* Replaces simint_create_zero_shell (shell.h:202, shell.c:297-302). */
void simint_create_zero_shell(struct simint_shell * G);

/* Replaces simint_initialize_multi_shellpair (shell.h:212, shell.c:305-309). */
void simint_initialize_multi_shellpair(struct simint_multi_shellpair * P);
/* Replaces simint_initialize_multi_shellpairs (shell.h:224, shell.c:312-316). */
void simint_initialize_multi_shellpairs(int n, struct simint_multi_shellpair * P);
/* Replaces simint_allocate_multi_shellpair (shell.h:238-241, shell.c:325-353). */
void simint_allocate_multi_shellpair(int na, struct simint_shell const * A,
                                     int nb, struct simint_shell const * B,
                                     struct simint_multi_shellpair * P,
                                     int screen_method);
/* Replaces simint_allocate_multi_shellpair2 (shell.h:252-254, shell.c:356-382). */
void simint_allocate_multi_shellpair2(int npair, struct simint_shell const * AB,
                                      struct simint_multi_shellpair * P,
                                      int screen_method);
/* Replaces simint_free_multi_shellpair (shell.h:261, shell.c:385-391). */
void simint_free_multi_shellpair(struct simint_multi_shellpair * P);
/* Replaces simint_free_multi_shellpairs (shell.h:271, shell.c:318-322). */
void simint_free_multi_shellpairs(int n, struct simint_multi_shellpair * P);
/* Replaces simint_fill_multi_shellpair (shell.h:288-291, shell.c:394-422). */
void simint_fill_multi_shellpair(int na, struct simint_shell const * A,
                                 int nb, struct simint_shell const * B,
                                 struct simint_multi_shellpair * P,
                                 int screen_method);
/* Replaces simint_fill_multi_shellpair2 (shell.h:311-313, shell.c:425-582). */
void simint_fill_multi_shellpair2(int npair, struct simint_shell const * AB,
                                  struct simint_multi_shellpair * P,
                                  int screen_method);
/* Replaces simint_create_multi_shellpair (shell.h:329-333, shell.c:585-592). */
void simint_create_multi_shellpair(int na, struct simint_shell const * A,
                                   int nb, struct simint_shell const * B,
                                   struct simint_multi_shellpair * P,
                                   int screen_method);
/* Replaces simint_create_multi_shellpair2 (shell.h:348-351, shell.c:595-602). */
void simint_create_multi_shellpair2(int npair, struct simint_shell const * AB,
                                    struct simint_multi_shellpair * P,
                                    int screen_method);
/* Replaces simint_cat_multi_shellpair (shell.h:363-366, shell.c:605-730). */
void simint_cat_multi_shellpair(int nmpair,
                                struct simint_multi_shellpair const ** Pin,
                                struct simint_multi_shellpair * Pout,
                                int screen_method);
/* Replaces simint_cat_shellpairs (shell.h:378-381, shell.c:733-873). */
void simint_cat_shellpairs(int nmpair,
                           struct simint_multi_shellpair const ** Pin,
                           struct simint_multi_shellpair * Pout,
                           int screen_method);

#ifdef __cplusplus
}
#endif
