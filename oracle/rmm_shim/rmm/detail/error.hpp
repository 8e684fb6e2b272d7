// Minimal stand-in for RMM's error header: the reference's bfs_thrust includes
// it but uses nothing from it.  Build-time shim for the reference runner only.
#pragma once
