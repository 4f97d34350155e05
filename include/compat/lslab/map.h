// The reference's include path <lslab/map.h> (depaulmillz/lslab,
// include/lslab/map.h), mapped onto this library's source-compatible front:
// callers written against lslab build unchanged with -I include/compat.
#pragma once
#include "../lslab_drop_in.h"
