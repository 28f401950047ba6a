// Serving loop (placeholder).
#include "ent_internal.h"
