// Stand-in for the reference's absent load_utils.cuh: the UltraGauss sources include it
// but call nothing from it. Used solely to compile the reference into oracle/_ref.
#pragma once
