// moderngpu header name the reference includes; the host restatement is in mgpu_host.hxx.
#pragma once
#include "mgpu_host.hxx"
