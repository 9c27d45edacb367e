#pragma once
/* Convenience header of the B200 Simint engine: pulls in the whole public
 * integral API (two- and one-electron), like the reference's
 * skel/simint/simint.h:1-7. */
#include "simint/ostei/ostei_config.h"
#include "simint/simint_init.h"
#include "simint/simint_eri.h"
#include "simint/simint_oneelectron.h"
#include "simint/shell/shell.h"
#include "simint/shell/shell_screen.h"
