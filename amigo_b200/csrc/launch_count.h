// Process-wide count of kernel launches made by this library (read through
// ab_launch_count); every launch site is followed by count_launch().
#pragma once

namespace ab {
void count_launch();
}
