// bion_file.h -- .bion files: reading every version the reference's loaders accept,
// writing the current one.
#pragma once
#include "common.h"

namespace bnc {
// Reads a .bion of version 3-14 into arrays this library owns (new[]; nuclei as
// 500-byte records), with the reference loader's migrations, validation and error codes
// (the BION_ERR_* values).  default_nuclei: a file without nucleus records gets one
// default nucleus per neuron, as both reference loaders create them; a checkpoint
// reload passes false, so a network saved without nuclei comes back without them.
int bion_read(const char* path, BncBionData* d, bool default_nuclei);
// Writes version 14 (bion_save, src/bion_loader_host.cpp:449-504).
int bion_write(const BncBionData& d, const char* path);
// Frees what bion_read (or a copy made the same way) allocated and zeroes *d.
void bion_free(BncBionData& d);
}  // namespace bnc
