// ingest.h -- movie files (multi-page TIFF, ETS) to u16 frames on the host.
#pragma once
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace gt {

// One opened movie: T frames of H x W pixels.  read_frame() is safe to call
// from several threads at once (positional reads only).
class MovieFile {
public:
    MovieFile();
    ~MovieFile();
    MovieFile(const MovieFile&) = delete;
    MovieFile& operator=(const MovieFile&) = delete;
    // 0 ok, 1 invalid file, 2 unsupported pixel format; *msg says why
    int open(const char* path, bool has_channel, uint32_t channel, std::string* msg);
    int read_frame(int t, uint16_t* out, std::string* msg) const;
    int T = 0, H = 0, W = 0;

private:
    struct Impl;
    Impl* impl;
};

// Channels of an ETS file with their frame counts, and its two dimensions.
int ets_channels(const char* path, std::vector<std::pair<uint32_t, int>>* chans, uint32_t dims[2], std::string* msg);

}  // namespace gt
