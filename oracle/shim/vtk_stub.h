// Stand-in types for the VTK writer in the reference's Domain.h.
// Test infrastructure: the PMG path never writes .vti files, so every call
// here is a no-op that only has to type-check.
#pragma once
#include <cstddef>
#define VTK_DOUBLE 11
template <typename T> struct vtkSmartPointer {
  T *p = nullptr;
  static vtkSmartPointer New() { return vtkSmartPointer{new T()}; }
  T *operator->() const { return p; }
};
struct vtkDataArrayStub {
  void SetNumberOfComponents(int) {}
  template <typename P> void SetArray(P *, std::size_t, int) {}
};
struct vtkDoubleArray : vtkDataArrayStub {};
struct vtkFloatArray : vtkDataArrayStub {};
struct vtkPointData {
  template <typename A> void SetScalars(const A &) {}
};
struct vtkImageData {
  vtkPointData pd;
  template <typename... A> void SetDimensions(A...) {}
  template <typename... A> void SetSpacing(A...) {}
  template <typename... A> void SetOrigin(A...) {}
  void AllocateScalars(int, int) {}
  vtkPointData *GetPointData() { return &pd; }
};
struct vtkXMLImageDataWriter {
  void SetFileName(const char *) {}
  template <typename A> void SetInputData(const A &) {}
  void Write() {}
};
