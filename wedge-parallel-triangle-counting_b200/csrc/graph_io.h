// graph_io.h -- host-side graph file parsing (see graph_io.cpp).
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/wetric.h"

namespace wetric {

// Parse a text edge list / Matrix Market body already in memory. Produces
// 0-based non-loop pairs and n = max id + 1. Returns a WETRIC_* status.
int parse_edge_text(const char *data, size_t size, bool matrix_market,
                    bool zero_indexed, std::vector<uint32_t> *src,
                    std::vector<uint32_t> *dst, uint64_t *n_out,
                    std::string *msg);

int parse_edge_file(const char *path, bool matrix_market, bool zero_indexed,
                    std::vector<uint32_t> *src, std::vector<uint32_t> *dst,
                    uint64_t *n_out, std::string *msg);

}  // namespace wetric
