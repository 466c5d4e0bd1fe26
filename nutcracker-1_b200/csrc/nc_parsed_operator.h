// An operator read from one of the file formats (YAML, protobuf): its unique
// sites, the 0-based sequence ordering them into the chain, and the chain's
// site array (pointing into the unique sites) handed out by
// nc_parsed_operator_sites.
#pragma once
#include <cstdint>
#include <vector>

#include "nutcracker_b200.h"

struct nc_parsed_operator {
    struct Site {
        uint32_t d = 0, cl = 0, cr = 0;
        std::vector<uint32_t> idx;     // (2,nnz) 1-based (from,to)
        std::vector<nc_complex> W;     // (d,d,nnz) column-major
    };
    std::vector<Site> unique;
    std::vector<uint32_t> sequence;
    std::vector<nc_operator_site> sites;

    // constructOperatorFrom (io.hpp:350-370): checks the sequence against the
    // unique sites and fills `sites`; throws nc::Error with the reference's messages.
    void assemble();
};
