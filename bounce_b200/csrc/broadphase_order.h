// Report order of a world broadphase query over static shape proxies.
#pragma once

#include <cstdint>

namespace b3g {

// rank[s] receives the position of shape s among the leaves that a world
// AABB query reports, for the proxies `lo`/`hi` (3 floats each per shape)
// inserted into the world's dynamic tree in shape order.  A contact's place
// in Bounce's contact lists follows that order: each new contact is pushed
// to the list's front as its shape is reported.
void query_report_ranks(const float (*lo)[3], const float (*hi)[3], uint32_t count, uint32_t* rank);

}  // namespace b3g
