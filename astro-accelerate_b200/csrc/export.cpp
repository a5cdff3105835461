// export.cpp -- DM-time output files (see export.hpp).
#include "export.hpp"

#include <cstdio>
#include <vector>

namespace aab200 {

size_t sd_per_file_from_file_size(size_t size_in_mb, size_t primary_dimension, size_t floats_per_element)
{
    if (primary_dimension == 0)
        return 0;
    const size_t nfloats = (size_in_mb * 1024 * 1024) / 4;
    return (nfloats * floats_per_element) / primary_dimension;
}

bool export_dd_data(int range, float ***data, size_t max_ntimesamples, const int *ndms, const int *in_bin,
                    const std::string &base, const int *ranges_to_export, int dms_per_file, std::string &err)
{
    for (int r = 0; r < range; ++r) {
        if (!ranges_to_export[r])
            continue;
        if (in_bin[r] < 1) {
            err = "inBin must be positive";
            return false;
        }
        const size_t nt = max_ntimesamples / static_cast<size_t>(in_bin[r]);
        const size_t ndm = static_cast<size_t>(ndms[r]);
        if (dms_per_file < 0)
            dms_per_file = static_cast<int>(ndm);
        if (dms_per_file == 0) {
            err = "DMs per file is 0 (a file smaller than one DM row)";
            return false;
        }
        std::vector<size_t> runs(ndm / static_cast<size_t>(dms_per_file), static_cast<size_t>(dms_per_file));
        if (ndm % static_cast<size_t>(dms_per_file))
            runs.push_back(ndm % static_cast<size_t>(dms_per_file));

        const std::string txt = base + "_" + std::to_string(r) + ".txt";
        FILE *ft = std::fopen(txt.c_str(), "w");
        if (!ft) {
            err = "cannot write " + txt;
            return false;
        }
        std::fprintf(ft, "%zu\n%zu\n%d\n%d\n", nt, ndm, dms_per_file, static_cast<int>(runs.size()));
        std::fclose(ft);

        std::vector<float> rows;
        size_t dm0 = 0;
        for (size_t i = 0; i < runs.size(); ++i) {
            rows.resize(runs[i] * nt);
            for (size_t d = 0; d < runs[i]; ++d)
                for (size_t t = 0; t < nt; ++t)
                    rows[d * nt + t] = data[r][dm0 + d][t];
            const std::string dat = base + "_" + std::to_string(r) + "_" + std::to_string(i) + ".dat";
            FILE *fd = std::fopen(dat.c_str(), "wb");
            if (!fd) {
                err = "cannot write " + dat;
                return false;
            }
            const bool ok = rows.empty() || std::fwrite(rows.data(), rows.size() * sizeof(float), 1, fd) == 1;
            std::fclose(fd);
            if (!ok) {
                err = "short write of " + dat;
                return false;
            }
            dm0 += runs[i];
        }
    }
    return true;
}

} // namespace aab200
