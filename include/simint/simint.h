#pragma once
/* Convenience header of the B200 Simint engine: pulls in the whole public
 * two-electron-integral API, like the reference's skel/simint/simint.h:1-7
 * (the one-electron part of the reference is not provided). */
#include "simint/ostei/ostei_config.h"
#include "simint/simint_init.h"
#include "simint/simint_eri.h"
#include "simint/shell/shell.h"
#include "simint/shell/shell_screen.h"
