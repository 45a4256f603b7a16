# TEST INFRASTRUCTURE ONLY: mechanical rewrite of the reference's CUDA C++
# for a host compiler (see host_shim.h); applied to copies in the build
# folder, never to the reference tree.
s/\r$//
s/extern __shared__ int sharedHash\[\];/int* sharedHash = host_shared_ints();/
s/([A-Za-z_][A-Za-z0-9_]*)<<<([^>]*)>>>\([[:space:]]*\)/launch_host(LaunchCfg(\2), \1)/g
s/([A-Za-z_][A-Za-z0-9_]*)<<<([^>]*)>>>\(/launch_host(LaunchCfg(\2), \1, /g
