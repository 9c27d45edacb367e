#pragma once
/* Schwarz screening values for shell pairs and primitive pairs. */
#include "simint/shell/shell.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces simint_shellscreen (skel/simint/shell/shell_screen.h:10-13). */
double simint_shellscreen(struct simint_shell const * A,
                          struct simint_shell const * B,
                          int screen_method);

/* Replaces simint_primscreen (skel/simint/shell/shell_screen.h:16-22). */
double simint_primscreen(struct simint_shell const * A,
                         struct simint_shell const * B,
                         double * out,
                         int screen_method);

/* Replaces simint_shellscreen_schwarz (shell_screen.h:26-28, shell_screen.c:48-83):
 * max |(ab|ab)| over all Cartesians, computed with the GPU ERI path. */
double simint_shellscreen_schwarz(struct simint_shell const * A,
                                  struct simint_shell const * B);

/* Replaces simint_shellscreen_fastschwarz (shell_screen.h:31-33, shell_screen.c:86-118). */
double simint_shellscreen_fastschwarz(struct simint_shell const * A,
                                      struct simint_shell const * B);

/* Replaces simint_primscreen_schwarz (shell_screen.h:40-43, shell_screen.c:127-223):
 * per primitive pair, max over diagonal Cartesians of |(ab|ab)| (no square
 * root: the tolerance is squared instead), padded like the pair arrays. */
double simint_primscreen_schwarz(struct simint_shell const * A,
                                 struct simint_shell const * B,
                                 double * out);

/* Replaces simint_primscreen_fastschwarz (shell_screen.h:51-54, shell_screen.c:227-270). */
double simint_primscreen_fastschwarz(struct simint_shell const * A,
                                     struct simint_shell const * B,
                                     double * out);

#ifdef __cplusplus
}
#endif
