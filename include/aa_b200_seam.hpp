/*
 * aa_b200_seam.hpp -- AstroAccelerate's dedispersion seam with the
 * reference's own C++ signatures, implemented by libaa_b200.so, so that code
 * written against the reference's runner compiles and links unchanged.
 *
 * Each declaration is the one of the reference header cited beside it, in
 * namespace astroaccelerate.  The buffers are the reference's: one unsigned
 * short per sample, [t][c] as loaded and [c][t] after the corner turn, rows
 * of i_nsamp = t_processed + maxshift/inBin samples (set by
 * set_dedispersion_constants), float DM-time rows [ndms][t_processed] out.
 *
 * Differences a caller may notice:
 *  - set_dedispersion_constants keeps its values per host thread (the
 *    reference writes __constant__ memory, shared by every thread of the
 *    process); dedisperse() reads the values its own thread set last;
 *  - d_dm_shifts is accepted and filled as the reference fills it, but the
 *    kernels read the host delay table `dmshifts`;
 *  - dedisperse() returns after its device work is complete (the
 *    reference's returns after the launch) and reports failures by its
 *    return value 1 with the reason in aa_b200_last_error().
 * The extern "C" twins aa_b200_seam_* in aa_b200.h take the same arguments.
 */
#ifndef AA_B200_SEAM_HPP
#define AA_B200_SEAM_HPP

#include <cstddef>

namespace astroaccelerate {

/* include/aa_device_load_data.hpp:15 (src/aa_device_load_data.cu:39-56) */
void load_chunk_data(unsigned short *device_pointer, unsigned short const *const host_pointer, int t_processed,
                     int maxshift, int nchans, float *dmshifts, float *d_dm_shifts, int nbits);
/* include/aa_device_load_data.hpp:17 (src/aa_device_load_data.cu:58-61) */
void set_dedispersion_constants(int t_processed, int maxshift);
/* include/aa_corner_turn.hpp:28 (src/aa_corner_turn.cpp:118-121) */
void corner_turn_SM_inplace(unsigned short *const d_input, unsigned short *const d_temporary,
                            const size_t primary_size, const size_t secondary_size);
/* include/aa_bin_gpu.hpp:17 (src/aa_bin_gpu.cpp:8-44) */
void bin_gpu(unsigned short *const d_input, float *const d_output, const int nchans, const int nsamp);
/* include/aa_dedisperse.hpp:20 (src/aa_dedisperse.cpp:5-163) */
int dedisperse(int i, int t_processed, int *inBin, float *dmshifts, unsigned short *d_input, float *d_output,
               float *d_dm_shifts, int nchans, float *tsamp, float *dm_low, float *dm_step, int const *const ndms,
               int nbits, int failsafe);
/* include/aa_device_save_data.hpp:12 (src/aa_device_save_data.cu:19-62) */
void save_data_offset_stream(int dm_range, int current_time_chunk, int **t_processed, long int inc, int *inBin,
                             int const *const ndms, float *d_DDTR_output, float ***output_buffer);

} // namespace astroaccelerate

#endif
