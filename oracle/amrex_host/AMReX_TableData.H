// Own host-only stand-in header: everything lives in AMReX_host.H.
#pragma once
#include "AMReX_host.H"
