// Stand-in for the reference's thread-to-core binding header (hwloc), which the engine header
// includes but the pattern operators do not use.  Test infrastructure only.
#pragma once
