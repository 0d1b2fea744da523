// fjb_launches.h -- process-wide count of this library's kernel launches.
#pragma once

namespace fjb {

// Called next to every kernel launch of the render path; read through
// fjb_kernel_launches().
void count_launch();

} // namespace fjb
