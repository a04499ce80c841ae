// fbp_host.hpp -- host-side set-up of the FBP path: the parts of the ctas
// CTrec constructor and Filter class that run once per reconstruction object
// (window, padding rule, angle table, physics coefficient).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace ctas {

// Error carrying a C-ABI status code; the ABI layer turns it into the return
// value and the thread's last-error message.
struct Error {
  int code;
  std::string msg;
};
[[noreturn]] void fail(int code, const std::string &msg);
// Message returned by ctas_fbp_last_error() on this thread.
void set_last_error(const std::string &msg);

int64_t padded_width(int64_t W);                       // lct.cpp:490
bool filter_known(int32_t ftype);
const char *filter_name(int32_t ftype);                // lct.cpp:93-109
int32_t filter_from_name(const std::string &name);     // lct.cpp:70-86 (throws)
void filter_check(int32_t ftype, float param);         // ct.h:144-152 (throws)
void filter_parse(const std::string &spec, int32_t *ftype, float *param);  // lct.cpp:236-248
int32_t contrast_from_name(const std::string &name);   // physical.world.cpp:19-27
const char *contrast_name(int32_t contrast);           // physical.world.cpp:43-54

// Filter::fill (lct.cpp:122-209) into `pixels` floats.
std::vector<float> filter_fill(int32_t ftype, float param, int64_t pixels);
// The CTrec window (lct.cpp:505-508).
std::vector<float> ctrec_window(int32_t ftype, float param, int64_t P, int64_t W,
                                int32_t contrast);

float arc_rad(float anarc, int64_t points);            // arcO lct.cpp:470-476
float step_rad(float anarc, int64_t points);           // angO lct.cpp:478-484
// cossins (lct.cpp:512-517): {sinf, cosf} pairs.
std::vector<float> angle_table(float arc_deg, int64_t N);
float rec_cof(float pixel_size, float lambda);         // lct.cpp:558-566

// Twiddle tables of the device FFT (2 P floats): per stage of the radix plan,
// (w^(m t), w^(4 m t)) for each butterfly index m, w = e^{-2 pi i / P},
// computed in double and rounded.
std::vector<float> fft_twiddles(int64_t P);
// Radix plan of the device FFT: stage radices from the largest block down.
std::vector<int> fft_radices(int64_t P);
// Position p of the device FFT's forward output holds frequency perm[p].
std::vector<int64_t> fft_output_order(int64_t P, const std::vector<int> &radices);

}  // namespace ctas

namespace ctas {
// Forms that write into caller-supplied storage and allocate nothing.
// scratch: P complex doubles; out: P floats.
void filter_fill_into(int32_t ftype, float param, int64_t P, float *out, void *scratch);
void angle_table_into(float arc_deg, int64_t N, float *tab);
void fft_twiddles_into(int64_t P, float *tw);
// Frequency held by position p of the device FFT's forward output.
int64_t fft_output_frequency(int64_t P, int64_t p);
}  // namespace ctas
