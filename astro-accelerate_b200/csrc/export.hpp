// export.hpp -- DM-time output files in the reference's Export_DD_data format
// (include/aa_pipeline_runner.hpp:165-216): per exported range r a text file
// <base>_<r>.txt holding nTimesamples, nDMs, DMs_per_file and the number of
// data files, one per line, and data files <base>_<r>_<i>.dat of float32
// [DMs in the file][nTimesamples], DM trials split into runs of DMs_per_file.
#pragma once

#include <cstddef>
#include <string>

namespace aab200 {

// include/aa_pipeline_runner.hpp:219-223: DM rows per file for a file size.
size_t sd_per_file_from_file_size(size_t size_in_mb, size_t primary_dimension, size_t floats_per_element);

// nTimesamples of range r = max_nTimesamples / inBin[r]; a negative
// DMs_per_file becomes the first exported range's DM count and stays so for
// later ranges (as the reference's parameter does).  Returns false with err
// set when a file cannot be written or DMs_per_file is 0.
bool export_dd_data(int range, float ***data, size_t max_ntimesamples, const int *ndms, const int *in_bin,
                    const std::string &base, const int *ranges_to_export, int dms_per_file, std::string &err);

} // namespace aab200
