/* gwycontainer.h -- opaque GwyContainer for the oracle build (test infrastructure). */
#ifndef SHIM_GWYCONTAINER_H
#define SHIM_GWYCONTAINER_H
#include <glib.h>
typedef struct _GwyContainer { gint dummy; } GwyContainer;
#endif
