/*
 * Project-written no-op stand-in for the few VTK 5 classes that the
 * reference's MRAG I/O headers name.  VTK is not installed in this image and
 * the oracle never writes VTK files; the classes only need to exist so that
 * the reference headers parse.  Every method does nothing.
 */
#pragma once
#include <stddef.h>
typedef long long vtkIdType;
#define VTK_PIXEL 8
#define VTK_VOXEL 11

class vtkObjectStub {
public:
    void Delete() { delete this; }
    virtual ~vtkObjectStub() {}
};

class vtkDataArrayStub : public vtkObjectStub {
    float dummy[1];
public:
    void SetName(const char *) {}
    void SetNumberOfComponents(int) {}
    void SetNumberOfTuples(vtkIdType) {}
    void *GetVoidPointer(vtkIdType) { return dummy; }
    int AddArray(vtkDataArrayStub *) { return 0; }
};

class vtkFloatArray : public vtkDataArrayStub {
public:
    static vtkFloatArray *New() { return new vtkFloatArray(); }
};

class vtkPoints : public vtkDataArrayStub {
public:
    static vtkPoints *New() { return new vtkPoints(); }
    void SetNumberOfPoints(vtkIdType) {}
};

class vtkPointData : public vtkDataArrayStub {};
class vtkCellData : public vtkDataArrayStub {};
class vtkCell : public vtkObjectStub {};

class vtkUnstructuredGrid : public vtkObjectStub {
    vtkPointData pd;
    vtkCellData cd;
public:
    static vtkUnstructuredGrid *New() { return new vtkUnstructuredGrid(); }
    void Allocate(vtkIdType = 0, vtkIdType = 0) {}
    void SetPoints(vtkPoints *) {}
    vtkIdType InsertNextCell(int, int, const vtkIdType *) { return 0; }
    vtkPointData *GetPointData() { return &pd; }
    vtkCellData *GetCellData() { return &cd; }
};

class vtkXMLUnstructuredGridWriter : public vtkObjectStub {
public:
    static vtkXMLUnstructuredGridWriter *New() { return new vtkXMLUnstructuredGridWriter(); }
    void SetFileName(const char *) {}
    void SetInput(vtkUnstructuredGrid *) {}
    int Write() { return 1; }
};
typedef vtkXMLUnstructuredGridWriter vtkUnstructuredGridWriter;
