// Environment-gated profiling rows, in the reference's format
// (crates/signinum-profile/src/lib.rs).
//
//   SIGNINUM_J2K_PROFILE_STAGES  per-call stage timings of the decode path
//                                (crates/signinum-j2k-native/src/profile.rs:16,
//                                the row of decode.rs:890-935)
//   SIGNINUM_GPU_ROUTE_PROFILE   one row per backend routing decision
//                                (crates/signinum-j2k-cuda/src/runtime.rs:19-130)
//
// Each variable is read once per process: "1", "true", "t", "yes", "y", "on",
// "enable", "enabled" (any case) emit one stderr row per event,
//   signinum_profile codec=<codec> op=<op> path=<path> key=value ...
// and "summary", "summaries", "aggregate", "aggregates" aggregate the events
// of a thread and print, when the thread ends, one row per distinct
// (codec, op, path, labels),
//   signinum_profile_summary codec=.. op=.. path=.. <labels> count=N <key>_sum=S [<key>_avg=A]
// with averages for timing fields (keys ending in _us, _ms, _ns).  Anything
// else, or an unset variable, disables them.
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace sgn {
namespace prof {

enum class Mode { Disabled, Rows, Summary };

// profile_stage_mode_from_value (signinum-profile lib.rs:55-88).
Mode mode_from_value(const char* value);
Mode stage_mode();  // SIGNINUM_J2K_PROFILE_STAGES, cached
Mode route_mode();  // SIGNINUM_GPU_ROUTE_PROFILE, cached

using Fields = std::vector<std::pair<std::string, std::string>>;

// format_profile_row.
std::string format_row(const char* codec, const char* op, const char* path, const Fields& fields);

// Stage rows: numeric fields, summarised with every field aggregated.
void emit_stages(const char* codec, const char* op, const char* path, const Fields& fields);
// Route rows: summarised as counts per route label (gpu_route_summary_labels:
// op as route_op, request, fmt, decision, reason, has_fast_packet,
// supports_output_format, hardware_decode).
void emit_route(const char* codec, const char* path, const Fields& fields);

}  // namespace prof
}  // namespace sgn
