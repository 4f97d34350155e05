// Declarations shared between the library's translation units (not part of
// the public C-ABI).
#pragma once

#include <cstdint>

#include "lsb.h"
#include "lsb_core.cuh"

void lsb_internal_map_view(const lsb_map* m, lsb::TableView* view, uint32_t* buckets);
// CUDA device the map's memory lives on.
int lsb_internal_map_device(const lsb_map* m);
// Lock mode a table was created with (LSB_LOCK_*).
uint32_t lsb_internal_lock_mode_map(const lsb_map* m);
uint32_t lsb_internal_lock_mode_set(const lsb_set* s);
