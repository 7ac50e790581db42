/*
 * Jacobian.hxx -- host-side Jacobian class with the reference's member names
 * (include/Jacobian.hxx:43-98).  setupDevice/toDevice/fromDevice go through
 * the solver context of the Platform; factor/sweep/solve are the device
 * phases of src/main.cxx:180-229.
 */
#ifndef TBS_JACOBIAN_HXX
#define TBS_JACOBIAN_HXX

#include "Mesh.hxx"

#include <cstdint>

class Jacobian {
  public:
    size_t nbytes = 0;

    int nvar = 0;
    int nelem = 0;
    int nintface = 0;

    std::vector<double> jacDLU;
    std::vector<double> jacD;
    std::vector<double> jacO1;
    std::vector<double> jacO2;
    std::vector<double> rhs;
    std::vector<double> res;
    std::vector<double> U;
    std::vector<double> U0;
    std::vector<double> dU;

    std::vector<double> A;
    std::vector<double> DinvC;

    std::string error;

    Jacobian() {}
    ~Jacobian() {}

    /* src/Jacobian.cxx:11-74 */
    bool fromFile(int nlineelem, const char *path = "gpuline.jacobian.data.bin");
    /* seeded synthetic values for a mesh (tbs_gen_jacobian) */
    bool fromGenerator(const Mesh &mesh, double shift, uint64_t seed);
    bool toFile(const char *path) const;

    /* src/Jacobian.cxx:76-117: packed in-line lower blocks A[e] */
    void assembleTriBlocks(Mesh &mesh);
    /* src/Jacobian.cxx:153-238, same resulting arrays */
    void resizeBlockSize(int nvar_new);

    /* src/Jacobian.cxx:240-290 */
    void setupDevice(Platform &gpu);
    void toDevice();
    void fromDevice();

  private:
    Platform *gpu_ = nullptr;
    void size_arrays(int nlineelem);
};

#endif /* TBS_JACOBIAN_HXX */
