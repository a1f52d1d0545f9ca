// ORACLE / TEST INFRASTRUCTURE ONLY.
// Compiles the reference's scene assembly (src/scene/scene_host.cpp) so its
// file-local light registration (addMeshTriangleLights, scene_host.cpp:77-106,
// then addStaticTriangleLights, :60-75, in the order assembleCornellScene and
// assembleGltfScene call them, :345-346, :413-414) can be applied to the
// host-compiled reference's scenes.  The asset loaders are not part of the
// traced path; they are stubbed.
#include "../src/scene/scene_host.cpp"

#include <stdexcept>

void wfref_register_lights(HostScene& scene) {
    addMeshTriangleLights(scene);
    addStaticTriangleLights(scene);
}

ObjScene loadObjScene(const char*) { throw std::runtime_error("asset loaders are not built into the host reference"); }
ObjMesh loadObjMesh(const char*) { throw std::runtime_error("asset loaders are not built into the host reference"); }
GltfScene loadGltfScene(const char*) { throw std::runtime_error("asset loaders are not built into the host reference"); }
