// Drop-in ImageAnalysis.hpp (the reference's ImageAnalysis.hpp:1-42): RGB
// histograms of exactly the requested graph output, counted on the GPU.
#pragma once

#include "RawEngine.hpp"

#include <array>
#include <cstdint>
#include <optional>
#include <vector>

namespace rawengine {

struct HistogramOptions {
    std::uint32_t bins = 256;   // 1..65536, equally spaced in [lower, upper]
    double lower = 0.0;
    double upper = 1.0;
};

struct ChannelHistogram {
    std::vector<std::uint64_t> counts;
    std::uint64_t underflow = 0, overflow = 0, nonfinite = 0;
    std::optional<float> minimum, maximum;   // all finite values, outliers included
};

struct RgbHistogram {
    RenderRequest request;
    HistogramOptions options;
    ImageDescriptor descriptor;
    std::uint64_t pixel_count = 0;
    std::array<ChannelHistogram, 3> channels;   // R, G, B in the output domain
};

// Bins are half-open except the last, which includes upper; signed values and
// headroom are not clipped; NaN and infinities count as non-finite and do not
// reach the extrema.  Nodes of this library are rendered on the device in
// bands of whole tile rows that stay in L2 and are counted there (counters in
// device memory, one read-back at the end); other nodes are rendered tile by
// tile as in the reference and each tile is counted on the device.
// Cancellation throws; callers never receive a partial result.
RAWENGINE_API RgbHistogram histogram_rgb(const Node& output, Rect source_bounds, const RenderRequest& request,
                                         const HistogramOptions& options = {},
                                         const CancellationToken* cancellation = nullptr);
RAWENGINE_API RgbHistogram histogram_rgb(const ImageGraph& graph, const RenderRequest& request,
                                         const HistogramOptions& options = {},
                                         const CancellationToken* cancellation = nullptr);

}  // namespace rawengine
