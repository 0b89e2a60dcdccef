// ref_state.h -- the in-memory series the reference build's shims read.
#pragma once

struct GrefSeries {
    int n = 0;
    int width = 0;
    int height = 0;
    bool is_tomo = false;
    const float* const* images = nullptr;  // n host images, width * height floats each
    const int* order = nullptr;            // processing order (zero tilt first)
    const float* tilts = nullptr;
    const char* const* names = nullptr;
    float* full_spectra = nullptr;         // optional n x (tile * tile)
};

GrefSeries& gref_series();
