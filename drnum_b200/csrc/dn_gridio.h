// Helpers of the .dnd restart format shared by the context entry points
// (dn_write_data / dn_read_data in dn_api.cu) and dn_gridio.cpp.
#pragma once

#include <cstddef>
#include <string>
#include "drnum_b200.h"

namespace dn {

std::string dnd_file_name(const char* base, int count);
void dnd_header(std::string& out, int prec, double time);
void dnd_values(std::string& out, int prec, const double* v, size_t n);
bool dnd_write_file(const std::string& name, const std::string& bytes);
bool dnd_read_file(const std::string& name, std::string& bytes);
bool dnd_parse_header(const std::string& bytes, int* prec, double* time, size_t* offset);
void dnd_get_values(const std::string& bytes, size_t offset, int prec, double* v, size_t n);

} // namespace dn
