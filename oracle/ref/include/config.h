/* Build shim: the reference's autotools config.h (Pipeline/hd/params.h:9).
 * HAVE_PSRDADA and HAVE_MPI stay undefined for the host build. */
#pragma once
