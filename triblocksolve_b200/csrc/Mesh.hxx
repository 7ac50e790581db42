/*
 * Mesh.hxx -- host-side Mesh and Platform classes with the reference's
 * member names (include/Mesh.hxx:27-67, include/Platform.hxx:25-93), built
 * on the C ABI of libtriblock.so.  Device buffers are owned by the solver
 * context (tbs_ctx) instead of per-array occa::memory members.
 */
#ifndef TBS_MESH_HXX
#define TBS_MESH_HXX

#include "../../include/triblock.h"

#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

/* Replaces Platform(comm, mode, device_id) (src/Platform.cxx:11-78).
 * Only compute_mode 2 (CUDA) exists in this build; any other mode throws. */
class Platform {
  public:
    int compute_mode;
    int device_id;
    tbs_ctx *ctx = nullptr;

    Platform(int compute_mode, int device_id);
    ~Platform();
    Platform(const Platform &) = delete;
    Platform &operator=(const Platform &) = delete;

    /* gpu.device.memoryAllocated() (src/main.cxx:97-99) */
    size_t memoryAllocated() const;
};

class Mesh {
  public:
    size_t nbytes = 0;

    int nvar = 0;
    int nelem = 0;
    int nintface = 0;
    int eftot = 0;

    int nline = 0;
    int nlineelem = 0;
    int max_line_nelem = 0;

    std::vector<int> epoint;
    std::vector<int> ef;
    std::vector<int> fc;

    std::vector<int> lines;
    std::vector<int> linesize;
    std::vector<int> lineface;
    std::vector<int> linepoint;

    std::string error;

    Mesh() {}
    ~Mesh() {}

    /* src/Mesh.cxx:11-73: read the stream-binary mesh (0-based in memory).
     * Returns false with `error` set instead of calling exit(1). */
    bool fromFile(const char *path = "gpuline.mesh.data.bin");
    /* structured L x K mesh in the reference's numbering */
    bool fromStructured(int L, int K, int nvar = 9);
    bool toFile(const char *path) const;

    /* src/Mesh.cxx:75-94 */
    void setupDevice(Platform &gpu);
    void toDevice();
    void fromDevice();

  private:
    Platform *gpu_ = nullptr;
    void finish_sizes();
};

#endif /* TBS_MESH_HXX */
