/* Hand-written public configuration for the oracle build of the reference. */
#pragma once
#define HMAT_VERSION "1.11.1-oracle"
