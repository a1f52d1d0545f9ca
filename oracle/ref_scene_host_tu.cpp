// ORACLE / TEST INFRASTRUCTURE ONLY.
// Compiles the reference's scene assembly (src/scene/scene_host.cpp) so its
// file-local light registration (addMeshTriangleLights, scene_host.cpp:77-106,
// then addStaticTriangleLights, :60-75, in the order assembleCornellScene and
// assembleGltfScene call them, :345-346, :413-414) can be applied to the
// host-compiled reference's scenes.  The asset loaders it calls are the
// reference's own (obj_loader.cpp, gltf_loader.cpp), built beside it.
#include "../src/scene/scene_host.cpp"

#include <stdexcept>

void wfref_register_lights(HostScene& scene) {
    addMeshTriangleLights(scene);
    addStaticTriangleLights(scene);
}

