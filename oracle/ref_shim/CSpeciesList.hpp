/* Shim for the species list of the absent carbon/state sources (test
 * infrastructure only): the flux code in the reference looks species up by
 * name and tests their flags; the oracle's driver fills state vectors
 * directly, so only these declarations are needed. */
#pragma once
#include <string>
#include <vector>
#include "carbon.h"

enum SpeciesFlags { SPECIES_NONE = 0, SPECIES_BOUNDARY = 1 << 0, SPECIES_KONSTANT = 1 << 2 };

struct CSpeciesList {
    std::vector<std::string> names;
    int index_of(const std::string &s) const {
        for (size_t k = 0; k < names.size(); ++k)
            if (names[k] == s) return (int)k;
        return -1;
    }
};
