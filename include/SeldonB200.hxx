// SeldonB200.hxx -- Seldon's sparse Krylov path on one B200 GPU.
//
// Include this header after Seldon's own (SeldonSolver.hxx, or Seldon.hxx
// with the iterative solvers) and link libseldon_b200.so.  A Seldon program
// moves its sparse system to the GPU by changing one template argument, the
// allocator, to CudaAlloc<double>:
//
//   typedef Matrix<double, General, RowSparse, CudaAlloc<double> > GpuMatrix;
//   typedef Vector<double, VectFull, CudaAlloc<double> > GpuVector;
//   GpuMatrix A;  A.Copy(A_host);          // upload a Seldon host matrix
//   GpuVector x(n), b;  Copy(b_host, b);   // host -> device
//   Iteration<double> iter(1000, 1e-10);
//   Preconditioner_Base M;
//   Cg(A, x, b, M, iter);                  // fused persistent CG on the GPU
//   Copy(x, x_host);                       // device -> host
//
// Everything below is an overload, a class specialisation or an allocator in
// namespace Seldon that C++ partial ordering prefers over Seldon's generic
// templates whenever the arguments are device types:
//
//   CudaAlloc<T>                              allocator concept of
//                                             share/Allocator.hxx:31-48
//   Vector<T, VectFull, CudaAlloc<T> >        vector/Vector.hxx:38-176
//   Matrix<double, Prop, RowSparse, CudaAlloc<double> >
//                                             matrix_sparse/Matrix_Sparse.hxx:42-195
//   Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >
//                                             matrix_sparse/Matrix_SymSparse.hxx:45-195
//   Mlt / MltAdd (NoTrans and SeldonTrans)    Functions_MatVect.cxx:72-130,
//                                             398-431, 526-564, 729-758, 915-927
//   Mlt(alpha, X), Add, Copy, DotProd, DotProdConj, Norm2
//                                             Functions_Vector.cxx:69-105,
//                                             240-246, 330-397, 540-549
//   SOR                                       Relaxation_MatVect.cxx:41-95, 176-298
//   Cg / BiCgStab / Gmres                     Cg.cxx:45-116, BiCgStab.cxx:43-145,
//                                             Gmres.cxx:44-183
//   Conjugate (no-op for real vectors)        Functions_Vector.hxx:351
//   JacobiPreconditioner<T>                   (absent from Seldon) z_i = r_i / A(i,i)
//
//   BiCg, BiCgcr, BiCgStabl, Cgne, Cgs,       BiCg.cxx:46-134, BiCgStabl.cxx:43-180,
//   CoCg, Gcr, Lsqr, MinRes, QCgs, QmrSym,    BiCgcr.cxx:44-118, Lsqr.cxx:40-135,
//   Symmlq, TfQmr                             QmrSym.cxx:41-165, Symmlq.cxx:45-161,
//                                             Cgne.cxx:40-127, Cgs.cxx:45-132,
//                                             CoCg.cxx:45-116, Gcr.cxx:45-141,
//                                             MinRes.cxx:46-153, QCgs.cxx:46-165,
//                                             TfQmr.cxx:44-243
//
// Seldon's other Krylov driver (Qmr) needs no overload: its generic
// template, instantiated on the device types, calls only the operations
// above, so every vector operation runs on the GPU.
//
// The solver overloads run the library's fused kernels when the
// preconditioner is Preconditioner_Base, JacobiPreconditioner or
// SorPreconditioner; with any other preconditioner class Seldon's own
// generic driver runs on the device types, every vector operation of it on
// the GPU.  The Iteration object is left in the state Seldon's driver leaves
// it in (iteration count, factor, error code) and the residual lines it
// prints are printed, from the device-side history, after the solve.
//
// Errors: a status from the library is thrown as a Seldon exception
// (share/Errors.hxx): NoMemory for a failed device allocation, WrongDim for
// inconsistent sizes or CSR arrays, WrongArgument for invalid arguments,
// Error otherwise.
//
// Work is queued on the stream set by Seldon::b200::SetStream (default: the
// legacy default stream); the scalar results (DotProd, Norm2, a solver's
// return) and every copy that touches host memory wait for it.
#ifndef SELDON_FILE_SELDON_B200_HXX
#define SELDON_FILE_SELDON_B200_HXX

#include <atomic>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "seldon_b200.h"

namespace Seldon
{

  namespace b200
  {
    inline void*& StreamSlot()
    {
      static thread_local void* s = 0;
      return s;
    }

    //! Stream (a cudaStream_t) on which this thread's device work is queued.
    inline void SetStream(void* stream) { StreamSlot() = stream; }
    inline void* GetStream() { return StreamSlot(); }

    //! Throws the Seldon exception matching a library status.
    inline void Check(int status, const std::string& function)
    {
      if (status == SB2_OK)
        return;
      std::string what = sb2_status_string(status);
      switch (status)
        {
        case SB2_ERR_NO_MEMORY:
          throw NoMemory(function, what);
        case SB2_ERR_INVALID_CSR:
          throw WrongDim(function, what);
        case SB2_ERR_INVALID_VALUE:
          throw WrongArgument(function, what);
        default:
          throw Error(function, what);
        }
    }

    inline unsigned long long NextSerial()
    {
      static std::atomic<unsigned long long> counter(0);
      return ++counter;
    }
  }


  /////////////////
  // CUDA MEMORY //
  /////////////////


  //! Allocator of device memory (the allocator concept of Allocator.hxx).
  /*! Device memory cannot be dereferenced on the host: the vector and matrix
    specialisations below are the only containers meant to use it. */
  template <class T>
  class CudaAlloc
  {
  public:
    typedef T value_type;
    typedef T* pointer;
    typedef const T* const_pointer;
    typedef T& reference;
    typedef const T& const_reference;

    pointer allocate(int num, void* h = 0)
    {
      void* p = 0;
      if (num > 0)
        b200::Check(sb2_device_alloc(sizeof(T) * size_t(num), &p),
                    "CudaAlloc::allocate");
      return static_cast<pointer>(p);
    }

    void deallocate(pointer data, int num, void* h = 0)
    {
      sb2_device_free(data);
    }

    //! New buffer of num entries; the old contents are not kept.
    void* reallocate(pointer data, int num, void* h = 0)
    {
      deallocate(data, num, h);
      return allocate(num, h);
    }

    //! Sets num bytes to c.
    void memoryset(pointer data, char c, size_t num)
    {
      if (num == 0)
        return;
      std::vector<char> buf(num, c);
      b200::Check(sb2_memcpy(data, &buf[0], num, b200::GetStream()),
                  "CudaAlloc::memoryset");
    }

    //! Copies num entries (device to device).
    void memorycpy(pointer datat, pointer datas, size_t num)
    {
      b200::Check(sb2_memcpy(datat, datas, num * sizeof(T), b200::GetStream()),
                  "CudaAlloc::memorycpy");
    }
  };


  namespace b200
  {
    template <class T>
    inline void FillValue(T* data, int n, const T& x)
    {
      if (n <= 0)
        return;
      std::vector<T> h(n, x);
      Check(sb2_memcpy(data, &h[0], sizeof(T) * size_t(n), GetStream()),
            "Vector::Fill");
    }

    inline void FillValue(double* data, int n, const double& x)
    {
      if (n > 0)
        Check(sb2_fill(n, x, data, GetStream()), "Vector::Fill");
    }
  }


  //////////////////////////
  // VECTOR ON THE DEVICE //
  //////////////////////////


  //! Dense vector whose entries live in device memory.
  /*! Same interface as Vector<T, VectFull, Allocator> (Vector.hxx:38-176)
    except element references: operator() returns the value, read from the
    device (one synchronous copy per call). */
  template <class T>
  class Vector<T, VectFull, CudaAlloc<T> >: public Vector_Base<T, CudaAlloc<T> >
  {
  public:
    typedef T value_type;
    typedef T* pointer;
    typedef const T* const_pointer;
    typedef T& reference;
    typedef const T& const_reference;
    typedef VectFull storage;

  private:
    typedef Vector_Base<T, CudaAlloc<T> > base;

  public:
    explicit Vector(): base() {}

    //! Allocates i entries (not initialised), as Seldon does.
    explicit Vector(int i): base(i)
    {
      this->data_ = this->vect_allocator_.allocate(i, this);
    }

    //! Takes ownership of a device buffer of i entries.
    Vector(int i, pointer data): base()
    {
      this->m_ = i;
      this->data_ = data;
    }

    Vector(const Vector<T, VectFull, CudaAlloc<T> >& X): base()
    {
      Copy(X);
    }

    ~Vector() {}

    void Clear()
    {
      if (this->data_ != NULL)
        this->vect_allocator_.deallocate(this->data_, this->m_);
      this->data_ = NULL;
      this->m_ = 0;
    }

    void Reallocate(int i)
    {
      if (i == this->m_)
        return;
      Clear();
      this->data_ = this->vect_allocator_.allocate(i, this);
      this->m_ = i;
    }

    //! Changes the length and keeps the first min(old, new) entries.
    void Resize(int i)
    {
      if (i == this->m_)
        return;
      pointer d = this->vect_allocator_.allocate(i, this);
      int keep = i < this->m_ ? i : this->m_;
      if (keep > 0)
        b200::Check(sb2_memcpy(d, this->data_, sizeof(T) * size_t(keep),
                               b200::GetStream()), "Vector::Resize");
      Clear();
      this->data_ = d;
      this->m_ = i;
    }

    //! Takes ownership of a device buffer of i entries.
    void SetData(int i, pointer data)
    {
      Clear();
      this->m_ = i;
      this->data_ = data;
    }

    //! Shares the buffer of V (call Nullify before either is destroyed).
    void SetData(const Vector<T, VectFull, CudaAlloc<T> >& V)
    {
      SetData(V.GetM(), V.GetData());
    }

    void Nullify()
    {
      this->m_ = 0;
      this->data_ = NULL;
    }

    //! Entry i, read from the device.
    value_type operator() (int i) const
    {
      T v;
      b200::Check(sb2_memcpy(&v, this->data_ + i, sizeof(T), b200::GetStream()),
                  "Vector::operator()");
      return v;
    }

    value_type Get(int i) const
    {
      return (*this)(i);
    }

    Vector<T, VectFull, CudaAlloc<T> >&
    operator= (const Vector<T, VectFull, CudaAlloc<T> >& X)
    {
      Copy(X);
      return *this;
    }

    void Copy(const Vector<T, VectFull, CudaAlloc<T> >& X)
    {
      if (&X == this)
        return;
      Reallocate(X.GetM());
      if (this->m_ > 0)
        b200::Check(sb2_memcpy(this->data_, X.GetData(),
                               sizeof(T) * size_t(this->m_), b200::GetStream()),
                    "Vector::Copy");
    }

    Vector<T, VectFull, CudaAlloc<T> > Copy() const
    {
      return Vector<T, VectFull, CudaAlloc<T> >(*this);
    }

    int GetDataSize() const
    {
      return this->m_;
    }

    void Zero()
    {
      b200::FillValue(this->data_, this->m_, T(0));
    }

    //! Entry i set to i (Vector.cxx Fill()).
    void Fill()
    {
      if (this->m_ <= 0)
        return;
      std::vector<T> h(this->m_);
      for (int i = 0; i < this->m_; i++)
        h[i] = T(i);
      b200::Check(sb2_memcpy(this->data_, &h[0], sizeof(T) * size_t(this->m_),
                             b200::GetStream()), "Vector::Fill");
    }

    template <class T0>
    void Fill(const T0& x)
    {
      b200::FillValue(this->data_, this->m_, T(x));
    }

    template <class T0>
    Vector<T, VectFull, CudaAlloc<T> >& operator= (const T0& x)
    {
      Fill(x);
      return *this;
    }

    template <class T0>
    Vector<T, VectFull, CudaAlloc<T> >& operator*= (const T0& alpha)
    {
      Mlt(alpha, *this);
      return *this;
    }

    //! Saves the entries in Seldon's binary format (Vector.cxx:848-870):
    //! the length first when with_size.
    void Write(std::string FileName, bool with_size = true) const
    {
      std::ofstream f(FileName.c_str(), std::ofstream::binary);
      if (!f.good())
        throw IOError("Vector::Write(string FileName, bool with_size)",
                      "Unable to open file \"" + FileName + "\".");
      std::vector<T> h(this->m_);
      if (this->m_ > 0)
        b200::Check(sb2_memcpy(&h[0], this->data_, sizeof(T) * size_t(this->m_),
                               b200::GetStream()), "Vector::Write");
      if (with_size)
        f.write(reinterpret_cast<const char*>(&this->m_), sizeof(int));
      f.write(reinterpret_cast<const char*>(h.data()), sizeof(T) * h.size());
      if (!f.good())
        throw IOError("Vector::Write(string FileName, bool with_size)", "Output operation failed.");
    }

    //! Loads a file in Seldon's binary format: the length from the file when
    //! with_size, else the vector's current length.
    void Read(std::string FileName, bool with_size = true)
    {
      std::ifstream f(FileName.c_str(), std::ifstream::binary);
      if (!f.good())
        throw IOError("Vector::Read(string FileName, bool with_size)",
                      "Unable to open file \"" + FileName + "\".");
      int m = this->m_;
      if (with_size)
        f.read(reinterpret_cast<char*>(&m), sizeof(int));
      if (!f.good() || m < 0)
        throw IOError("Vector::Read(string FileName, bool with_size)", "Invalid length.");
      std::vector<T> h(m);
      f.read(reinterpret_cast<char*>(h.data()), sizeof(T) * h.size());
      if (!f.good())
        throw IOError("Vector::Read(string FileName, bool with_size)",
                      "Input operation failed: the file holds fewer values.");
      Reallocate(m);
      if (m > 0)
        b200::Check(sb2_memcpy(this->data_, h.data(), sizeof(T) * size_t(m), b200::GetStream()),
                    "Vector::Read");
    }

    //! Seldon's host vector holding these entries (read back from the device).
    Vector<T, VectFull> HostCopy() const
    {
      Vector<T, VectFull> h(this->m_);
      if (this->m_ > 0)
        b200::Check(sb2_memcpy(h.GetData(), this->data_, sizeof(T) * size_t(this->m_),
                               b200::GetStream()), "Vector::HostCopy");
      return h;
    }

    //! Takes the length and entries of a host vector.
    template <class Allocator0>
    void Upload(const Vector<T, VectFull, Allocator0>& h)
    {
      Reallocate(h.GetM());
      if (this->m_ > 0)
        b200::Check(sb2_memcpy(this->data_, h.GetData(), sizeof(T) * size_t(this->m_),
                               b200::GetStream()), "Vector::Upload");
    }

    //! Largest absolute value and its index, as Vector::GetNormInf and
    //! GetNormInfIndex compute them (Vector.cxx:765-800), on the entries
    //! read back from the device: for inspection, not for loops.
    value_type GetNormInf() const
    {
      return HostCopy().GetNormInf();
    }

    int GetNormInfIndex() const
    {
      return HostCopy().GetNormInfIndex();
    }

    //! Seldon's FillRand values (drawn on the host), then uploaded.
    void FillRand()
    {
      Vector<T, VectFull> h(this->m_);
      h.FillRand();
      Upload(h);
    }

    //! Seldon's text format (Vector::WriteText / ReadText), through a host copy.
    void WriteText(std::string FileName) const
    {
      HostCopy().WriteText(FileName);
    }

    void WriteText(std::ostream& FileStream) const
    {
      HostCopy().WriteText(FileStream);
    }

    void ReadText(std::string FileName)
    {
      Vector<T, VectFull> h;
      h.ReadText(FileName);
      Upload(h);
    }

    void ReadText(std::istream& FileStream)
    {
      Vector<T, VectFull> h;
      h.ReadText(FileStream);
      Upload(h);
    }

    //! One entry added at the end (Vector::Append, PushBack): the buffer is
    //! reallocated, so build long vectors on the host and copy them instead.
    void Append(const T& x)
    {
      const int m = this->m_;
      Resize(m + 1);
      b200::Check(sb2_memcpy(this->data_ + m, &x, sizeof(T), b200::GetStream()),
                  "Vector::Append");
    }

    template <class T0>
    void PushBack(const T0& x)
    {
      Append(T(x));
    }

    //! The entries of X (host or device) added at the end.
    template <class Allocator0>
    void PushBack(const Vector<T, VectFull, Allocator0>& X)
    {
      const int m = this->m_;
      Resize(m + X.GetM());
      if (X.GetM() > 0)
        b200::Check(sb2_memcpy(this->data_ + m, X.GetData(), sizeof(T) * size_t(X.GetM()),
                               b200::GetStream()), "Vector::PushBack");
    }

    //! Prints the entries (read back from the device) as Vector::Print does.
    void Print() const
    {
      std::vector<T> h(this->m_);
      if (this->m_ > 0)
        b200::Check(sb2_memcpy(&h[0], this->data_, sizeof(T) * size_t(this->m_),
                               b200::GetStream()), "Vector::Print");
      for (int i = 0; i < this->m_; i++)
        std::cout << h[i] << '\t';
      std::cout << std::endl;
    }
  };


  ////////////////////////////
  // MATRICES ON THE DEVICE //
  ////////////////////////////


  namespace b200
  {
    //! Device CSR matrix behind the RowSparse and RowSymSparse
    //! specialisations: an opaque library handle that owns device copies
    //! of ptr_/ind_/data_ (and the SpMV layouts built from them).
    //! Device scratch released on scope exit.
    struct DeviceBuffer
    {
      void* p;
      explicit DeviceBuffer(size_t bytes): p(NULL)
      {
        Check(sb2_device_alloc(bytes, &p), "sb2_device_alloc");
      }
      ~DeviceBuffer()
      {
        sb2_device_free(p);
      }
    private:
      DeviceBuffer(const DeviceBuffer&);
      DeviceBuffer& operator= (const DeviceBuffer&);
    };

    //! The Seldon host type a device matrix downloads into.
    template <int Symmetric> struct HostMatrix
    {
      typedef Matrix<double, General, RowSparse> type;
    };
    template <> struct HostMatrix<1>
    {
      typedef Matrix<double, Symmetric, RowSymSparse> type;
    };

    template <int Symmetric>
    class DeviceCsr: public Matrix_Base<double, CudaAlloc<double> >
    {
    protected:
      sb2_csr* h_;
      int nz_;
      unsigned long long serial_;

    public:
      DeviceCsr(): h_(0), nz_(0), serial_(0)
      {
        this->m_ = 0;
        this->n_ = 0;
        this->data_ = NULL;
      }

      DeviceCsr(const DeviceCsr& A): h_(0), nz_(0), serial_(0)
      {
        this->m_ = 0;
        this->n_ = 0;
        this->data_ = NULL;
        CopyDevice(A);
      }

      ~DeviceCsr()
      {
        if (h_)
          sb2_csr_destroy(h_);
      }

      DeviceCsr& operator= (const DeviceCsr& A)
      {
        CopyDevice(A);
        return *this;
      }

      //! Builds the device matrix from host CSR arrays (copied, not kept).
      void Create(int i, int j, int nz, const int* ptr, const int* ind,
                  const double* val)
      {
        std::vector<int> zero_ptr;
        if (ptr == NULL)
          {
            zero_ptr.assign(i + 1, 0);
            ptr = &zero_ptr[0];
          }
        sb2_csr* h = 0;
        Check(sb2_csr_create(i, j, nz, ptr, ind, val, Symmetric, 1, &h),
              "Matrix::SetData");
        if (h_)
          sb2_csr_destroy(h_);
        h_ = h;
        this->m_ = i;
        this->n_ = j;
        nz_ = nz;
        serial_ = NextSerial();
      }

      //! i x j matrix without entries (Matrix_Sparse(i, j)).
      void Reallocate(int i, int j)
      {
        Create(i, j, 0, NULL, NULL, NULL);
      }

      //! Takes the host vectors' contents and leaves them empty, as
      //! Matrix_Sparse::SetData does (Matrix_Sparse.cxx:305-415).
      template <class Storage0, class Allocator0, class Storage1,
                class Allocator1, class Storage2, class Allocator2>
      void SetData(int i, int j, Vector<double, Storage0, Allocator0>& values,
                   Vector<int, Storage1, Allocator1>& ptr,
                   Vector<int, Storage2, Allocator2>& ind)
      {
        if (ptr.GetM() != i + 1)
          throw WrongDim("Matrix::SetData", "ptr must have i+1 entries");
        if (ind.GetM() != values.GetM())
          throw WrongDim("Matrix::SetData", "ind and values sizes differ");
        Create(i, j, values.GetM(), ptr.GetData(), ind.GetData(),
               values.GetData());
        values.Clear();
        ptr.Clear();
        ind.Clear();
      }

      //! Takes host arrays allocated with malloc/calloc (Seldon's default
      //! allocators): they are copied to the device and freed.
      void SetData(int i, int j, int nz, double* values, int* ptr, int* ind)
      {
        Create(i, j, nz, ptr, ind, values);
        free(values);
        free(ptr);
        free(ind);
      }

      void Clear()
      {
        if (h_)
          sb2_csr_destroy(h_);
        h_ = 0;
        nz_ = 0;
        this->m_ = 0;
        this->n_ = 0;
        serial_ = NextSerial();
      }

      //! Stored entries (the upper triangle for RowSymSparse).
      int GetNonZeros() const { return nz_; }
      int GetDataSize() const { return nz_; }
      //! Lengths of ptr and ind (Matrix_Sparse.cxx:1018-1037).
      int GetPtrSize() const { return this->m_ + 1; }
      int GetIndSize() const { return nz_; }

      //! Element (i, j) by the reference's lookup (Matrix_Sparse.cxx:
      //! 1054-1083; RowSymSparse reads (min, max) in the upper triangle,
      //! Matrix_SymSparse.cxx:1013-1053).  Each call downloads the stored
      //! arrays: it is for inspection, not for loops.
      double operator() (int i, int j) const
      {
        CheckIndex(i, j, "Matrix::operator()");
        std::vector<int> ptr, ind;
        std::vector<double> val;
        Download(ptr, ind, val);
        return Lookup(ptr, ind, val, i, j);
      }

      //! The dense matrix, row by row (Matrix_Sparse::Print,
      //! Matrix_Sparse.cxx:1491-1499), from one download.
      void Print() const
      {
        std::vector<int> ptr, ind;
        std::vector<double> val;
        Download(ptr, ind, val);
        for (int i = 0; i < this->m_; i++)
          {
            for (int j = 0; j < this->n_; j++)
              std::cout << Lookup(ptr, ind, val, i, j) << "\t";
            std::cout << std::endl;
          }
      }

      //! Library handle (for the C ABI of seldon_b200.h).
      sb2_csr* GetHandle() const
      {
        if (!h_)
          throw WrongArgument("Matrix::GetHandle", "matrix not initialised");
        return h_;
      }

      //! Changes every time the device matrix is rebuilt.
      unsigned long long GetSerial() const { return serial_; }

      //! Host copies of the stored arrays.
      void Download(std::vector<int>& ptr, std::vector<int>& ind,
                    std::vector<double>& val) const
      {
        ptr.assign(this->m_ + 1, 0);
        ind.resize(nz_);
        val.resize(nz_);
        if (!h_)
          return;
        Check(sb2_csr_download(h_, &ptr[0], nz_ ? &ind[0] : NULL,
                               nz_ ? &val[0] : NULL), "Matrix::Download");
      }

      //! Saves the stored arrays in Seldon's binary format (Matrix_Sparse.cxx:
      //! 1531-1556; RowSymSparse writes the row count for n): a Seldon program
      //! can Read the file back into a host matrix.
      void Write(std::string FileName) const
      {
        std::ofstream f(FileName.c_str(), std::ofstream::binary);
        if (!f.good())
          throw IOError("Matrix::Write(string FileName)",
                        "Unable to open file \"" + FileName + "\".");
        std::vector<int> p, i;
        std::vector<double> v;
        Download(p, i, v);
        int head[3] = {this->m_, Symmetric ? this->m_ : this->n_, nz_};
        f.write(reinterpret_cast<const char*>(head), sizeof(head));
        f.write(reinterpret_cast<const char*>(p.data()), sizeof(int) * p.size());
        f.write(reinterpret_cast<const char*>(i.data()), sizeof(int) * i.size());
        f.write(reinterpret_cast<const char*>(v.data()), sizeof(double) * v.size());
        if (!f.good())
          throw IOError("Matrix::Write(string FileName)", "Output operation failed.");
      }

      //! Loads a file in Seldon's binary format (Matrix_Sparse.cxx:1650-1680)
      //! into the device matrix.
      void Read(std::string FileName)
      {
        std::ifstream f(FileName.c_str(), std::ifstream::binary);
        if (!f.good())
          throw IOError("Matrix::Read(string FileName)",
                        "Unable to open file \"" + FileName + "\".");
        int head[3] = {0, 0, 0};
        f.read(reinterpret_cast<char*>(head), sizeof(head));
        if (!f.good() || head[0] < 0 || head[1] < 0 || head[2] < 0)
          throw IOError("Matrix::Read(string FileName)", "Invalid header.");
        std::vector<int> p(head[0] + 1), i(head[2]);
        std::vector<double> v(head[2]);
        f.read(reinterpret_cast<char*>(p.data()), sizeof(int) * p.size());
        f.read(reinterpret_cast<char*>(i.data()), sizeof(int) * i.size());
        f.read(reinterpret_cast<char*>(v.data()), sizeof(double) * v.size());
        if (!f.good())
          throw IOError("Matrix::Read(string FileName)",
                        "Input operation failed: the file is shorter than its header says.");
        Create(head[0], head[1], head[2], p.data(), i.empty() ? NULL : i.data(),
               v.empty() ? NULL : v.data());
      }

      //! Builds the matrix on the device from DEVICE triplets, as
      //! ConvertMatrix_from_Coordinates fills it (Matrix_Conversions.cxx:
      //! 1291-1334 RowSparse, 1397-1467 RowSymSparse; sb2_coo_to_csr).
      void AssembleDevice(int nnz, const int* row, const int* col,
                          const double* val, int index)
      {
        int m = 0, n = 0, nz = 0;
        int *p = NULL, *i = NULL;
        double* v = NULL;
        Check(sb2_coo_to_csr(nnz, row, col, val, index, this->m_, this->n_,
                             Symmetric, GetStream(), &m, &n, &nz, &p, &i, &v),
              "ConvertMatrix_from_Coordinates");
        sb2_csr* h = 0;
        int st = sb2_csr_create(m, n, nz, p, i, v, Symmetric, 1, &h);
        sb2_device_free(p);
        sb2_device_free(i);
        sb2_device_free(v);
        Check(st, "ConvertMatrix_from_Coordinates");
        if (h_)
          sb2_csr_destroy(h_);
        h_ = h;
        this->m_ = m;
        this->n_ = n;
        nz_ = nz;
        serial_ = NextSerial();
      }

      //! The same from HOST triplets (copied to the device first).
      void AssembleHost(int nnz, const int* row, const int* col,
                        const double* val, int index)
      {
        DeviceBuffer r(sizeof(int) * size_t(nnz)), c(sizeof(int) * size_t(nnz)),
          v(sizeof(double) * size_t(nnz));
        if (nnz > 0)
          {
            Check(sb2_memcpy(r.p, row, sizeof(int) * size_t(nnz), GetStream()), "upload");
            Check(sb2_memcpy(c.p, col, sizeof(int) * size_t(nnz), GetStream()), "upload");
            Check(sb2_memcpy(v.p, val, sizeof(double) * size_t(nnz), GetStream()), "upload");
          }
        AssembleDevice(nnz, static_cast<const int*>(r.p), static_cast<const int*>(c.p),
                       static_cast<const double*>(v.p), index);
      }

      //! Reads "row column value" lines (1-based) as Matrix_Sparse::ReadText
      //! does (Matrix_Sparse.cxx:1692-1724, ReadCoordinateMatrix 1885-1980),
      //! then assembles the matrix on the device.
      void ReadText(std::string FileName)
      {
        std::ifstream f(FileName.c_str());
        if (!f.is_open())
          throw IOError("Matrix_Sparse::ReadText(string FileName)",
                        std::string("Unable to open file \"") + FileName + "\".");
        std::vector<int> r, c;
        std::vector<double> v;
        int row = 0, col = 0;
        double entry = 0.0;
        while (!f.eof())
          {
            f >> row >> col >> entry;
            if (f.fail())
              break;
            if (row < 1)
              throw IOError("ReadCoordinateMatrix",
                            "Error : Row number should be greater than 0 but is equal to "
                            + to_str(row));
            if (col < 1)
              throw IOError("ReadCoordinateMatrix",
                            "Error : Column number should be greater than 0 but is equal to "
                            + to_str(col));
            r.push_back(row);
            c.push_back(col);
            v.push_back(entry);
          }
        Clear();
        if (!r.empty())
          AssembleHost(int(r.size()), &r[0], &c[0], &v[0], 1);
      }

      //! Writes "row column value" lines as Matrix_Sparse::WriteText does
      //! (Matrix_Sparse.cxx:1568-1616): Seldon's own writer on a host copy,
      //! so the text is the same byte for byte.
      void WriteText(std::string FileName) const
      {
        typename HostMatrix<Symmetric>::type A;
        DownloadTo(A);
        A.WriteText(FileName);
      }

    protected:
      void CheckIndex(int i, int j, const char* function) const
      {
#ifdef SELDON_CHECK_BOUNDS
        if (i < 0 || i >= this->m_)
          throw WrongRow(function, "row index out of range");
        if (j < 0 || j >= this->n_)
          throw WrongCol(function, "column index out of range");
#endif
      }

      //! The reference's element lookup on downloaded arrays: scan row i
      //! while k < b-1 and ind[k] < j, then test ind[k] == j.
      static double Lookup(const std::vector<int>& ptr, const std::vector<int>& ind,
                           const std::vector<double>& val, int i, int j)
      {
        if (Symmetric && i > j)
          std::swap(i, j);
        const int a = ptr[i], b = ptr[i + 1];
        if (a == b)
          return 0.0;
        int k = a;
        while (k < b - 1 && ind[k] < j)
          k++;
        return ind[k] == j ? val[k] : 0.0;
      }

      void CopyDevice(const DeviceCsr& A)
      {
        if (&A == this)
          return;
        if (!A.h_)
          {
            Clear();
            return;
          }
        std::vector<int> p, i;
        std::vector<double> v;
        A.Download(p, i, v);
        Create(A.GetM(), A.GetN(), A.nz_, &p[0], i.empty() ? NULL : &i[0],
               v.empty() ? NULL : &v[0]);
      }

      template <class MatrixHost>
      void UploadFrom(const MatrixHost& A)
      {
        Create(A.GetM(), A.GetN(), A.GetNonZeros(), A.GetPtr(), A.GetInd(),
               A.GetData());
      }

      template <class MatrixHost>
      void DownloadTo(MatrixHost& A) const
      {
        std::vector<int> p, i;
        std::vector<double> v;
        Download(p, i, v);
        Vector<double> values(nz_);
        Vector<int> ptr(this->m_ + 1), ind(nz_);
        for (int k = 0; k < nz_; k++)
          {
            values(k) = v[k];
            ind(k) = i[k];
          }
        for (int k = 0; k <= this->m_; k++)
          ptr(k) = p[k];
        A.SetData(this->m_, this->n_, values, ptr, ind);
      }
    };
  }


  //! General CSR matrix in device memory (Matrix<T, Prop, RowSparse>).
  template <class Prop>
  class Matrix<double, Prop, RowSparse, CudaAlloc<double> >:
    public b200::DeviceCsr<0>
  {
  public:
    typedef double value_type;
    typedef Prop property;
    typedef RowSparse storage;
    typedef CudaAlloc<double> allocator;

    Matrix() {}

    Matrix(int i, int j)
    {
      this->Reallocate(i, j);
    }

    template <class Storage0, class Allocator0, class Storage1,
              class Allocator1, class Storage2, class Allocator2>
    Matrix(int i, int j, Vector<double, Storage0, Allocator0>& values,
           Vector<int, Storage1, Allocator1>& ptr,
           Vector<int, Storage2, Allocator2>& ind)
    {
      this->SetData(i, j, values, ptr, ind);
    }

    //! Device-to-device copy.
    void Copy(const Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A)
    {
      this->CopyDevice(A);
    }

    //! Upload of a Seldon host matrix (its arrays are left as they are).
    template <class Prop0, class Allocator0>
    void Copy(const Matrix<double, Prop0, RowSparse, Allocator0>& A)
    {
      this->UploadFrom(A);
    }

    //! Download into a Seldon host matrix.
    template <class Prop0, class Allocator0>
    void CopyToHost(Matrix<double, Prop0, RowSparse, Allocator0>& A) const
    {
      this->DownloadTo(A);
    }
  };


  //! Symmetric matrix in device memory, upper triangle stored
  //! (Matrix<T, Prop, RowSymSparse>).
  template <class Prop>
  class Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >:
    public b200::DeviceCsr<1>
  {
  public:
    typedef double value_type;
    typedef Prop property;
    typedef RowSymSparse storage;
    typedef CudaAlloc<double> allocator;

    Matrix() {}

    Matrix(int i, int j)
    {
      this->Reallocate(i, j);
    }

    template <class Storage0, class Allocator0, class Storage1,
              class Allocator1, class Storage2, class Allocator2>
    Matrix(int i, int j, Vector<double, Storage0, Allocator0>& values,
           Vector<int, Storage1, Allocator1>& ptr,
           Vector<int, Storage2, Allocator2>& ind)
    {
      this->SetData(i, j, values, ptr, ind);
    }

    void Copy(const Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A)
    {
      this->CopyDevice(A);
    }

    template <class Prop0, class Allocator0>
    void Copy(const Matrix<double, Prop0, RowSymSparse, Allocator0>& A)
    {
      this->UploadFrom(A);
    }

    template <class Prop0, class Allocator0>
    void CopyToHost(Matrix<double, Prop0, RowSymSparse, Allocator0>& A) const
    {
      this->DownloadTo(A);
    }
  };


  ///////////////////////////////////
  // ASSEMBLY FROM COORDINATE FORM //
  ///////////////////////////////////


  //! ConvertMatrix_from_Coordinates (Matrix_Conversions.cxx:1291-1334) with
  //! the triplets in device memory: sorted and assembled on the device.  The
  //! triplet vectors are emptied, as Seldon empties them.
  template <class Prop>
  void ConvertMatrix_from_Coordinates(Vector<int, VectFull, CudaAlloc<int> >& IndRow,
                                      Vector<int, VectFull, CudaAlloc<int> >& IndCol,
                                      Vector<double, VectFull, CudaAlloc<double> >& Val,
                                      Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
                                      int index = 0)
  {
    if (IndCol.GetM() != IndRow.GetM() || Val.GetM() != IndRow.GetM())
      throw WrongDim("ConvertMatrix_from_Coordinates", "triplet vectors differ in length");
    A.AssembleDevice(IndRow.GetM(), IndRow.GetData(), IndCol.GetData(), Val.GetData(), index);
    IndRow.Clear();
    IndCol.Clear();
    Val.Clear();
  }


  //! RowSymSparse form (Matrix_Conversions.cxx:1397-1467): entries below the
  //! diagonal are dropped.
  template <class Prop>
  void ConvertMatrix_from_Coordinates(Vector<int, VectFull, CudaAlloc<int> >& IndRow,
                                      Vector<int, VectFull, CudaAlloc<int> >& IndCol,
                                      Vector<double, VectFull, CudaAlloc<double> >& Val,
                                      Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
                                      int index = 0)
  {
    if (IndRow.GetM() <= 0)
      return;
    if (IndCol.GetM() != IndRow.GetM() || Val.GetM() != IndRow.GetM())
      throw WrongDim("ConvertMatrix_from_Coordinates", "triplet vectors differ in length");
    A.AssembleDevice(IndRow.GetM(), IndRow.GetData(), IndCol.GetData(), Val.GetData(), index);
    IndRow.Clear();
    IndCol.Clear();
    Val.Clear();
  }


  //! Copy(ArrayRowSparse -> RowSparse) (Matrix_Conversions.cxx:3843-3857)
  //! into a device matrix: Seldon's own flattening of the rows, which are
  //! already sorted and merged, then one upload.
  template <class T0, class Prop0, class Allocator0, class Prop1>
  void Copy(const Matrix<T0, Prop0, ArrayRowSparse, Allocator0>& A,
            Matrix<double, Prop1, RowSparse, CudaAlloc<double> >& B)
  {
    Matrix<double, General, RowSparse> h;
    Copy(A, h);
    B.Copy(h);
  }


  //! Copy(ArrayRowSymSparse -> RowSymSparse) (Matrix_Conversions.cxx:
  //! 3859-3875) into a device matrix.
  template <class T0, class Prop0, class Allocator0, class Prop1>
  void Copy(const Matrix<T0, Prop0, ArrayRowSymSparse, Allocator0>& A,
            Matrix<double, Prop1, RowSymSparse, CudaAlloc<double> >& B)
  {
    Matrix<double, Symmetric, RowSymSparse> h;
    Copy(A, h);
    B.Copy(h);
  }


  //! Host triplets into a device matrix: copied to the device, then
  //! assembled there.
  template <class Prop, class Alloc1, class Alloc2, class Alloc3>
  void ConvertMatrix_from_Coordinates(Vector<int, VectFull, Alloc1>& IndRow,
                                      Vector<int, VectFull, Alloc2>& IndCol,
                                      Vector<double, VectFull, Alloc3>& Val,
                                      Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
                                      int index = 0)
  {
    if (IndCol.GetM() != IndRow.GetM() || Val.GetM() != IndRow.GetM())
      throw WrongDim("ConvertMatrix_from_Coordinates", "triplet vectors differ in length");
    A.AssembleHost(IndRow.GetM(), IndRow.GetData(), IndCol.GetData(), Val.GetData(), index);
    IndRow.Clear();
    IndCol.Clear();
    Val.Clear();
  }


  template <class Prop, class Alloc1, class Alloc2, class Alloc3>
  void ConvertMatrix_from_Coordinates(Vector<int, VectFull, Alloc1>& IndRow,
                                      Vector<int, VectFull, Alloc2>& IndCol,
                                      Vector<double, VectFull, Alloc3>& Val,
                                      Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
                                      int index = 0)
  {
    if (IndRow.GetM() <= 0)
      return;
    if (IndCol.GetM() != IndRow.GetM() || Val.GetM() != IndRow.GetM())
      throw WrongDim("ConvertMatrix_from_Coordinates", "triplet vectors differ in length");
    A.AssembleHost(IndRow.GetM(), IndRow.GetData(), IndCol.GetData(), Val.GetData(), index);
    IndRow.Clear();
    IndCol.Clear();
    Val.Clear();
  }


  ////////////
  // BLAS-1 //
  ////////////


  //! X = alpha X (Functions_Vector.cxx:69-74).
  template <class T0>
  void Mlt(const T0& alpha, Vector<double, VectFull, CudaAlloc<double> >& X)
  {
    b200::Check(sb2_scal(X.GetM(), double(alpha), X.GetData(), b200::GetStream()),
                "Mlt(alpha, X)");
  }

  //! Y = Y + alpha X; nothing when alpha is zero (Functions_Vector.cxx:85-105).
  template <class T0>
  void Add(const T0& alpha, const Vector<double, VectFull, CudaAlloc<double> >& X,
           Vector<double, VectFull, CudaAlloc<double> >& Y)
  {
    if (double(alpha) == 0.0)
      return;
    if (X.GetM() != Y.GetM())
      throw WrongDim("Add(alpha, X, Y)", "X and Y sizes differ");
    b200::Check(sb2_axpy(X.GetM(), double(alpha), X.GetData(), Y.GetData(),
                         b200::GetStream()), "Add(alpha, X, Y)");
  }

  //! Y = X, Y resized (Functions_Vector.cxx:240-246).
  inline void Copy(const Vector<double, VectFull, CudaAlloc<double> >& X,
                   Vector<double, VectFull, CudaAlloc<double> >& Y)
  {
    Y.Copy(X);
  }

  //! Host vector to device vector.
  template <class Allocator0>
  void Copy(const Vector<double, VectFull, Allocator0>& X,
            Vector<double, VectFull, CudaAlloc<double> >& Y)
  {
    Y.Reallocate(X.GetM());
    if (X.GetM() > 0)
      b200::Check(sb2_memcpy(Y.GetData(), X.GetData(), sizeof(double) * size_t(X.GetM()),
                             b200::GetStream()), "Copy(host, device)");
  }

  //! Device vector to host vector.
  template <class Allocator0>
  void Copy(const Vector<double, VectFull, CudaAlloc<double> >& X,
            Vector<double, VectFull, Allocator0>& Y)
  {
    Y.Reallocate(X.GetM());
    if (X.GetM() > 0)
      b200::Check(sb2_memcpy(Y.GetData(), X.GetData(), sizeof(double) * size_t(X.GetM()),
                             b200::GetStream()), "Copy(device, host)");
  }

  //! Host index vector to device vector (device triplets for assembly).
  template <class Allocator0>
  void Copy(const Vector<int, VectFull, Allocator0>& X,
            Vector<int, VectFull, CudaAlloc<int> >& Y)
  {
    Y.Reallocate(X.GetM());
    if (X.GetM() > 0)
      b200::Check(sb2_memcpy(Y.GetData(), X.GetData(), sizeof(int) * size_t(X.GetM()),
                             b200::GetStream()), "Copy(host, device)");
  }

  //! Device index vector to host vector.
  template <class Allocator0>
  void Copy(const Vector<int, VectFull, CudaAlloc<int> >& X,
            Vector<int, VectFull, Allocator0>& Y)
  {
    Y.Reallocate(X.GetM());
    if (X.GetM() > 0)
      b200::Check(sb2_memcpy(Y.GetData(), X.GetData(), sizeof(int) * size_t(X.GetM()),
                             b200::GetStream()), "Copy(device, host)");
  }

  //! Real vectors are their own conjugate (Functions_Vector.hxx:351).
  inline void Conjugate(Vector<double, VectFull, CudaAlloc<double> >&)
  {
  }

  //! Sum of X_i Y_i (Functions_Vector.cxx:330-346), deterministic order.
  inline double DotProd(const Vector<double, VectFull, CudaAlloc<double> >& X,
                        const Vector<double, VectFull, CudaAlloc<double> >& Y)
  {
    if (X.GetM() != Y.GetM())
      throw WrongDim("DotProd(X, Y)", "X and Y sizes differ");
    double r = 0.0;
    b200::Check(sb2_dot(X.GetM(), X.GetData(), Y.GetData(), &r, b200::GetStream()),
                "DotProd(X, Y)");
    return r;
  }

  //! Real vectors: DotProdConj is DotProd (Functions_Vector.cxx:391-397).
  inline double DotProdConj(const Vector<double, VectFull, CudaAlloc<double> >& X,
                            const Vector<double, VectFull, CudaAlloc<double> >& Y)
  {
    return DotProd(X, Y);
  }

  //! Unscaled 2-norm sqrt(sum X_i^2) (Functions_Vector.cxx:540-549).
  inline double Norm2(const Vector<double, VectFull, CudaAlloc<double> >& X)
  {
    double r = 0.0;
    b200::Check(sb2_nrm2(X.GetM(), X.GetData(), &r, b200::GetStream()), "Norm2(X)");
    return r;
  }


  ////////////
  // SPMV   //
  ////////////


  namespace b200
  {
    template <class MatrixD>
    void SpMV(const MatrixD& M, int trans, double alpha,
              const Vector<double, VectFull, CudaAlloc<double> >& X, double beta,
              Vector<double, VectFull, CudaAlloc<double> >& Y, bool overwrite)
    {
      const int nx = trans ? M.GetM() : M.GetN();
      const int ny = trans ? M.GetN() : M.GetM();
      if (X.GetM() != nx || Y.GetM() != ny)
        throw WrongDim("MltAdd(alpha, M, X, beta, Y)",
                       "vector sizes do not match the matrix");
      if (overwrite)
        Check(sb2_mlt(M.GetHandle(), trans, alpha, X.GetData(), Y.GetData(),
                      GetStream()), "Mlt(M, X, Y)");
      else
        Check(sb2_spmv(M.GetHandle(), trans, alpha, X.GetData(), beta,
                       Y.GetData(), GetStream()), "MltAdd(alpha, M, X, beta, Y)");
    }
  }


  //! Y = beta Y + alpha M X (Functions_MatVect.cxx:398-431).
  template <class T0, class Prop1, class T3>
  void MltAdd(const T0 alpha,
              const Matrix<double, Prop1, RowSparse, CudaAlloc<double> >& M,
              const Vector<double, VectFull, CudaAlloc<double> >& X,
              const T3 beta, Vector<double, VectFull, CudaAlloc<double> >& Y)
  {
    b200::SpMV(M, 0, double(alpha), X, double(beta), Y, false);
  }

  //! Symmetric, upper triangle stored (Functions_MatVect.cxx:526-564).
  template <class T0, class Prop1, class T3>
  void MltAdd(const T0 alpha,
              const Matrix<double, Prop1, RowSymSparse, CudaAlloc<double> >& M,
              const Vector<double, VectFull, CudaAlloc<double> >& X,
              const T3 beta, Vector<double, VectFull, CudaAlloc<double> >& Y)
  {
    b200::SpMV(M, 0, double(alpha), X, double(beta), Y, false);
  }

  //! Y = beta Y + alpha op(M) X (Functions_MatVect.cxx:729-758, 915-927).
  //! One overload per transposition flag class, as Seldon declares them
  //! (Functions_MatVect.hxx:230-350), so that these are the exact matches.
#define SELDON_B200_MLTADD_TRANS(FLAG, STORAGE)                                \
  template <class T0, class Prop1, class T3>                                    \
  void MltAdd(const T0 alpha, const FLAG& Trans,                                \
              const Matrix<double, Prop1, STORAGE, CudaAlloc<double> >& M,      \
              const Vector<double, VectFull, CudaAlloc<double> >& X,            \
              const T3 beta, Vector<double, VectFull, CudaAlloc<double> >& Y)   \
  {                                                                             \
    b200::SpMV(M, Trans.NoTrans() ? 0 : 1, double(alpha), X, double(beta), Y,  \
               false);                                                          \
  }

  SELDON_B200_MLTADD_TRANS(SeldonTranspose, RowSparse)
  SELDON_B200_MLTADD_TRANS(SeldonTranspose, RowSymSparse)
  SELDON_B200_MLTADD_TRANS(class_SeldonNoTrans, RowSparse)
  SELDON_B200_MLTADD_TRANS(class_SeldonNoTrans, RowSymSparse)
  SELDON_B200_MLTADD_TRANS(class_SeldonTrans, RowSparse)
  SELDON_B200_MLTADD_TRANS(class_SeldonTrans, RowSymSparse)
  SELDON_B200_MLTADD_TRANS(class_SeldonConjTrans, RowSparse)
  SELDON_B200_MLTADD_TRANS(class_SeldonConjTrans, RowSymSparse)

#undef SELDON_B200_MLTADD_TRANS

  //! Y = M X (Functions_MatVect.cxx:72-83: Y.Fill(0), then MltAdd).
  template <class Prop1>
  void Mlt(const Matrix<double, Prop1, RowSparse, CudaAlloc<double> >& M,
           const Vector<double, VectFull, CudaAlloc<double> >& X,
           Vector<double, VectFull, CudaAlloc<double> >& Y)
  {
    b200::SpMV(M, 0, 1.0, X, 0.0, Y, true);
  }

  template <class Prop1>
  void Mlt(const Matrix<double, Prop1, RowSymSparse, CudaAlloc<double> >& M,
           const Vector<double, VectFull, CudaAlloc<double> >& X,
           Vector<double, VectFull, CudaAlloc<double> >& Y)
  {
    b200::SpMV(M, 0, 1.0, X, 0.0, Y, true);
  }

  //! Y = alpha M X (Functions_MatVect.cxx:98-109).
  template <class Prop1>
  void Mlt(const double& alpha,
           const Matrix<double, Prop1, RowSparse, CudaAlloc<double> >& M,
           const Vector<double, VectFull, CudaAlloc<double> >& X,
           Vector<double, VectFull, CudaAlloc<double> >& Y)
  {
    b200::SpMV(M, 0, alpha, X, 0.0, Y, true);
  }

  template <class Prop1>
  void Mlt(const double& alpha,
           const Matrix<double, Prop1, RowSymSparse, CudaAlloc<double> >& M,
           const Vector<double, VectFull, CudaAlloc<double> >& X,
           Vector<double, VectFull, CudaAlloc<double> >& Y)
  {
    b200::SpMV(M, 0, alpha, X, 0.0, Y, true);
  }

  //! Y = op(M) X (Functions_MatVect.cxx:121-130).
  template <class Prop1>
  void Mlt(const SeldonTranspose& Trans,
           const Matrix<double, Prop1, RowSparse, CudaAlloc<double> >& M,
           const Vector<double, VectFull, CudaAlloc<double> >& X,
           Vector<double, VectFull, CudaAlloc<double> >& Y)
  {
    b200::SpMV(M, Trans.NoTrans() ? 0 : 1, 1.0, X, 0.0, Y, true);
  }

  template <class Prop1>
  void Mlt(const SeldonTranspose& Trans,
           const Matrix<double, Prop1, RowSymSparse, CudaAlloc<double> >& M,
           const Vector<double, VectFull, CudaAlloc<double> >& X,
           Vector<double, VectFull, CudaAlloc<double> >& Y)
  {
    b200::SpMV(M, Trans.NoTrans() ? 0 : 1, 1.0, X, 0.0, Y, true);
  }


  /////////
  // SOR //
  /////////


  //! Sweeps of (S)SOR on A X = B, bit-identical to the sequential sweeps
  //! (Relaxation_MatVect.cxx:41-95).  type_ssor: 0 symmetric, 2 forward,
  //! 3 backward.
  template <class Prop0, class T3>
  void SOR(const Matrix<double, Prop0, RowSparse, CudaAlloc<double> >& A,
           Vector<double, VectFull, CudaAlloc<double> >& X,
           const Vector<double, VectFull, CudaAlloc<double> >& B,
           const T3& omega, int iter, int type_ssor = 2)
  {
    b200::Check(sb2_sor(A.GetHandle(), X.GetData(), B.GetData(), double(omega), iter,
                        type_ssor, b200::GetStream()), "SOR");
  }

  //! Symmetric storage (Relaxation_MatVect.cxx:176-298).
  template <class Prop0, class T3>
  void SOR(const Matrix<double, Prop0, RowSymSparse, CudaAlloc<double> >& A,
           Vector<double, VectFull, CudaAlloc<double> >& X,
           const Vector<double, VectFull, CudaAlloc<double> >& B,
           const T3& omega, int iter, int type_ssor = 2)
  {
    b200::Check(sb2_sor(A.GetHandle(), X.GetData(), B.GetData(), double(omega), iter,
                        type_ssor, b200::GetStream()), "SOR");
  }


  ////////////////////
  // PRECONDITIONERS //
  ////////////////////


  //! Jacobi preconditioner z_i = r_i / A(i,i) (absent from Seldon; same
  //! Solve/TransSolve interface as Preconditioner_Base, Iterative.hxx:24-39).
  /*! The diagonal is looked up as Matrix_Sparse::operator()(i, i) does: the
    first stored entry of row i with column i; a row without one gives a
    division by zero.  Usable with host matrices (Seldon's element access)
    and with device matrices (library kernel, diagonal cached per matrix). */
  template <class T>
  class JacobiPreconditioner
  {
    sb2_precond* h_;
    unsigned long long serial_;

  public:
    JacobiPreconditioner(): h_(0), serial_(0) {}
    JacobiPreconditioner(const JacobiPreconditioner&): h_(0), serial_(0) {}
    JacobiPreconditioner& operator= (const JacobiPreconditioner&)
    {
      Release();
      return *this;
    }
    ~JacobiPreconditioner() { Release(); }

    void Release()
    {
      if (h_)
        sb2_precond_destroy(h_);
      h_ = 0;
      serial_ = 0;
    }

    //! Library handle for device matrix A (created once per matrix).
    template <class MatrixD>
    const sb2_precond* GetHandle(const MatrixD& A)
    {
      if (!h_ || serial_ != A.GetSerial())
        {
          Release();
          b200::Check(sb2_precond_create(A.GetHandle(), SB2_PRECOND_JACOBI, 1.0, 1,
                                         1, &h_), "JacobiPreconditioner");
          serial_ = A.GetSerial();
        }
      return h_;
    }

    //! Host matrices and vectors: z_i = r_i / A(i,i).
    template <class Matrix1, class Vector1>
    void Solve(const Matrix1& A, const Vector1& r, Vector1& z)
    {
      for (int i = 0; i < r.GetM(); i++)
        z(i) = r(i) / A(i, i);
    }

    template <class Matrix1, class Vector1>
    void TransSolve(const Matrix1& A, const Vector1& r, Vector1& z)
    {
      Solve(A, r, z);
    }

    template <class Prop1>
    void Solve(const Matrix<double, Prop1, RowSparse, CudaAlloc<double> >& A,
               const Vector<double, VectFull, CudaAlloc<double> >& r,
               Vector<double, VectFull, CudaAlloc<double> >& z)
    {
      DeviceSolve(A, r, z);
    }

    template <class Prop1>
    void Solve(const Matrix<double, Prop1, RowSymSparse, CudaAlloc<double> >& A,
               const Vector<double, VectFull, CudaAlloc<double> >& r,
               Vector<double, VectFull, CudaAlloc<double> >& z)
    {
      DeviceSolve(A, r, z);
    }

    template <class Prop1>
    void TransSolve(const Matrix<double, Prop1, RowSparse, CudaAlloc<double> >& A,
                    const Vector<double, VectFull, CudaAlloc<double> >& r,
                    Vector<double, VectFull, CudaAlloc<double> >& z)
    {
      DeviceSolve(A, r, z);
    }

    template <class Prop1>
    void TransSolve(const Matrix<double, Prop1, RowSymSparse, CudaAlloc<double> >& A,
                    const Vector<double, VectFull, CudaAlloc<double> >& r,
                    Vector<double, VectFull, CudaAlloc<double> >& z)
    {
      DeviceSolve(A, r, z);
    }

  private:
    template <class MatrixD>
    void DeviceSolve(const MatrixD& A,
                     const Vector<double, VectFull, CudaAlloc<double> >& r,
                     Vector<double, VectFull, CudaAlloc<double> >& z)
    {
      b200::Check(sb2_precond_solve(GetHandle(A), r.GetData(), z.GetData(),
                                    b200::GetStream()), "JacobiPreconditioner::Solve");
    }
  };


  /////////////
  // SOLVERS //
  /////////////


  namespace b200
  {
    //! Reads and writes the protected state of Iteration<Titer>
    //! (Iterative.hxx:47-108) that its public interface does not expose.
    template <class Titer>
    struct IterationState: public Iteration<Titer>
    {
      static int MaxIter(const Iteration<Titer>& it)
      {
        return it.*(&IterationState::max_iter);
      }
      static int PrintLevel(const Iteration<Titer>& it)
      {
        return it.*(&IterationState::print_level);
      }
      static void SetFactor(Iteration<Titer>& it, Titer f)
      {
        it.*(&IterationState::facteur_reste) = f;
      }
    };

    //! Reads the parameters of Seldon's SorPreconditioner (Precond_Ssor.cxx:24-90).
    template <class T>
    struct SorState: public SorPreconditioner<T>
    {
      static bool Symmetric(const SorPreconditioner<T>& M)
      {
        return M.*(&SorState::symmetric_precond);
      }
      static int NbIter(const SorPreconditioner<T>& M)
      {
        return M.*(&SorState::nb_iter);
      }
      static T Omega(const SorPreconditioner<T>& M)
      {
        return M.*(&SorState::omega);
      }
    };

    //! Device handle of a preconditioner, released at scope exit.
    struct PrecondHandle
    {
      sb2_precond* owned;
      const sb2_precond* use;
      PrecondHandle(): owned(0), use(0) {}
      ~PrecondHandle()
      {
        if (owned)
          sb2_precond_destroy(owned);
      }
    };

    //! Preconditioners the fused solvers run natively.
    template <class P>
    struct PrecondTraits
    {
      static const bool native = false;
      template <class MatrixD>
      static void Acquire(P&, const MatrixD&, PrecondHandle&) {}
    };

    template <>
    struct PrecondTraits<Preconditioner_Base>
    {
      static const bool native = true;
      template <class MatrixD>
      static void Acquire(Preconditioner_Base&, const MatrixD&, PrecondHandle&) {}
    };

    template <class T>
    struct PrecondTraits<JacobiPreconditioner<T> >
    {
      static const bool native = true;
      template <class MatrixD>
      static void Acquire(JacobiPreconditioner<T>& M, const MatrixD& A,
                          PrecondHandle& h)
      {
        h.use = M.GetHandle(A);
      }
    };

    template <class T>
    struct PrecondTraits<SorPreconditioner<T> >
    {
      static const bool native = true;
      template <class MatrixD>
      static void Acquire(SorPreconditioner<T>& M, const MatrixD& A,
                          PrecondHandle& h)
      {
        Check(sb2_precond_create(A.GetHandle(), SB2_PRECOND_SOR,
                                 double(SorState<T>::Omega(M)),
                                 SorState<T>::NbIter(M),
                                 SorState<T>::Symmetric(M) ? 1 : 0, &h.owned),
              "SorPreconditioner");
        h.use = h.owned;
      }
    };

    enum SolverKind
    {
      kCg, kBiCgStab, kGmres, kGmresCgs2, kCgs, kTfQmr, kMinRes, kGcr, kBiCgStabl, kQCgs,
      kBiCg, kCoCg, kCgne, kBiCgcr, kLsqr, kQmrSym, kSymmlq
    };

    inline const char* BreakdownMessage(SolverKind kind, int code)
    {
      // the strings Cg.cxx:82,101, BiCgStab.cxx:77,87,107, Cgs.cxx:80,110,
      // TfQmr.cxx:116,138,148,186,219, MinRes.cxx:120,142, Gcr.cxx:108,
      // BiCgStabl.cxx:99,115, QCgs.cxx:86,108,138, BiCg.cxx:86,115 and
      // CoCg.cxx:84,102, Cgne.cxx:90,110, BiCgcr.cxx:85,101 and
      // Lsqr.cxx:88,100,108 and QmrSym.cxx:83,95,114,121,140 pass to Fail
      if (kind == kCg)
        return code == 1 ? "Cg breakdown #1" : "Cg breakdown #2";
      if (kind == kCgs)
        return code == 1 ? "Cgs breakdown #1" : "Cgs breakdown #2";
      if (kind == kMinRes)
        return code == 1 ? "Minres breakdown #1" : "MinRes breakdown #2";
      if (kind == kGcr)
        return "Gcr breakdown #1";
      if (kind == kBiCgStabl)
        return code == 1 ? "Bicgstabl breakdown #1" : "Bicgstabl Breakdown #2";
      if (kind == kBiCg)
        return code == 1 ? "Bicg breakdown #1" : "Bicg breakdown #2";
      if (kind == kCoCg)
        return code == 1 ? "Cocg breakdown #1" : "Cocg breakdown #2";
      if (kind == kCgne)
        return code == 1 ? "Cgne breakdown #1" : "Cgne breakdown #2";
      if (kind == kBiCgcr)
        return code == 1 ? "Bicgcr breakdown #1" : "Bicgcr breakdown #2";
      if (kind == kLsqr)
        return code == 1 ? "Lsqr breakdown #1"
                         : (code == 2 ? "Lsqr breakdown #2" : "Lsqr breakdown #3");
      if (kind == kQmrSym)
        {
          static const char* const qmr[] = {"Qmr breakdown #1", "Qmr breakdown #2",
                                            "Qmr breakdown #3", "Qmr breakdown #4",
                                            "Qmr breakdown #5"};
          return qmr[code == 1 ? 0 : (code >= 3 && code <= 6 ? code - 2 : 4)];
        }
      if (kind == kQCgs)
        return code == 1 ? "QCgs breakdown #1"
                         : (code == 2 ? "Qcgs breakdown #2" : "Qcgs breakdown #3");
      if (kind == kTfQmr)
        {
          if (code == 1)
            return "Tfqmr breakdown: sigma=0";
          if (code == 2)
            return "Tfqmr breakdown: alpha=0";
          return code == 5 ? "tfqmr breakdown: beta=0" : "Tfqmr breakdown: tau=0";
        }
      if (code == 1)
        return "Bicgstab breakdown #1";
      return code == 2 ? "Bicgstab breakdown #2" : "Bicgstab breakdown #3";
    }

    //! Runs one fused solver and leaves `iter` as Seldon's driver would.
    template <class Titer, class MatrixD, class P>
    int RunSolver(SolverKind kind, MatrixD& A,
                  Vector<double, VectFull, CudaAlloc<double> >& x,
                  const Vector<double, VectFull, CudaAlloc<double> >& b,
                  P& M, Iteration<Titer>& iter)
    {
      const int N = A.GetM();
      if (N <= 0)
        return 0;
      if (x.GetM() != N || b.GetM() != N)
        throw WrongDim("Iterative solver", "x and b must have A.GetM() entries");
      PrecondHandle ph;
      PrecondTraits<P>::Acquire(M, A, ph);
      sb2_iter_params prm;
      prm.tol = double(iter.GetTolerance());
      prm.max_iter = IterationState<Titer>::MaxIter(iter);
      prm.restart = iter.GetRestart();
      prm.print_level = IterationState<Titer>::PrintLevel(iter);
      prm.init_guess_null = iter.IsInitGuess_Null() ? 1 : 0;
      int cap = 0;
      std::vector<double> hist;
      std::vector<int> hist_it;
      if (prm.print_level >= 1)
        {
          cap = 2 * (prm.max_iter > 0 ? prm.max_iter : 0) + 8;
          hist.resize(cap);
          hist_it.resize(cap);
        }
      sb2_iter_result res;
      int st;
      if (kind == kCg)
        st = sb2_cg(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                    cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap, GetStream());
      else if (kind == kBiCgStab)
        st = sb2_bicgstab(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                          cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap,
                          GetStream());
      else if (kind == kGmres)
        st = sb2_gmres(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                       cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap,
                       GetStream());
      else if (kind == kCgs)
        st = sb2_cgs(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                     cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap, GetStream());
      else if (kind == kTfQmr)
        st = sb2_tfqmr(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                       cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap,
                       GetStream());
      else if (kind == kMinRes)
        st = sb2_minres(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                        cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap,
                        GetStream());
      else if (kind == kGcr)
        st = sb2_gcr(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                     cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap, GetStream());
      else if (kind == kBiCgStabl)
        st = sb2_bicgstabl(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                           cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap,
                           GetStream());
      else if (kind == kQCgs)
        st = sb2_qcgs(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                      cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap, GetStream());
      else if (kind == kBiCg)
        st = sb2_bicg(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                      cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap, GetStream());
      else if (kind == kCoCg)
        st = sb2_cocg(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                      cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap, GetStream());
      else if (kind == kCgne)
        st = sb2_cgne(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                      cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap, GetStream());
      else if (kind == kBiCgcr)
        st = sb2_bicgcr(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                        cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap, GetStream());
      else if (kind == kLsqr)
        st = sb2_lsqr(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                      cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap, GetStream());
      else if (kind == kQmrSym)
        st = sb2_qmrsym(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                        cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap, GetStream());
      else if (kind == kSymmlq)
        st = sb2_symmlq(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                        cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap, GetStream());
      else
        st = sb2_gmres_cgs2(A.GetHandle(), ph.use, x.GetData(), b.GetData(), &prm, &res,
                            cap ? &hist[0] : NULL, cap ? &hist_it[0] : NULL, cap,
                            GetStream());
      static const char* const names[] = {"Cg", "BiCgStab", "Gmres", "Gmres", "Cgs", "TfQmr",
                                          "MinRes", "Gcr", "BiCgStabl", "QCgs", "BiCg",
                                          "CoCg", "Cgne", "BiCgcr", "Lsqr", "QmrSym",
                                          "Symmlq"};
      Check(st, names[kind]);
      // Init() found a zero right-hand side: Seldon returns at once
      if (res.init_failed)
        return iter.ErrorCode();
      IterationState<Titer>::SetFactor(iter, Titer(res.facteur_reste));
      // the lines Iteration::Finished prints (Iterative.cxx:282-287)
      for (int k = 0; k < res.hist_len && k < cap; k++)
        {
          const int it = hist_it[k];
          if ((prm.print_level >= 1 && it % 100 == 0) || prm.print_level >= 6)
            std::cout << "Residu at iteration number " << it << "  "
                      << Titer(hist[k]) << std::endl;
        }
      iter.SetNumberIteration(res.nb_iter);
      if (res.error_code > 0)
        iter.Fail(res.error_code, BreakdownMessage(kind, res.error_code));
      return iter.ErrorCode();
    }
  }


  namespace b200
  {
    //! Fused kernels for the preconditioners of PrecondTraits; Seldon's
    //! generic driver (on the device types) for any other class.
    template <bool native>
    struct Dispatch
    {
      template <class Titer, class MatrixD, class P>
      static int Run(SolverKind kind, MatrixD& A,
                     Vector<double, VectFull, CudaAlloc<double> >& x,
                     const Vector<double, VectFull, CudaAlloc<double> >& b,
                     P& M, Iteration<Titer>& iter)
      {
        return RunSolver(kind, A, x, b, M, iter);
      }
    };

    template <>
    struct Dispatch<false>
    {
      template <class Titer, class MatrixD, class P>
      static int Run(SolverKind kind, MatrixD& A,
                     Vector<double, VectFull, CudaAlloc<double> >& x,
                     const Vector<double, VectFull, CudaAlloc<double> >& b,
                     P& M, Iteration<Titer>& iter)
      {
        typedef Vector<double, VectFull, CudaAlloc<double> > VectorD;
        if (kind == kCg)
          return Seldon::Cg<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kBiCgStab)
          return Seldon::BiCgStab<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kCgs)
          return Seldon::Cgs<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kTfQmr)
          return Seldon::TfQmr<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kMinRes)
          return Seldon::MinRes<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kGcr)
          return Seldon::Gcr<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kBiCgStabl)
          return Seldon::BiCgStabl<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kQCgs)
          return Seldon::QCgs<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kBiCg)
          return Seldon::BiCg<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kCoCg)
          return Seldon::CoCg<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kCgne)
          return Seldon::Cgne<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kBiCgcr)
          return Seldon::BiCgcr<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kLsqr)
          return Seldon::Lsqr<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kQmrSym)
          return Seldon::QmrSym<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        if (kind == kSymmlq)
          return Seldon::Symmlq<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
        return Seldon::Gmres<Titer, MatrixD, VectorD, P>(A, x, b, M, iter);
      }
    };

    template <class Titer, class MatrixD, class P>
    int Solve(SolverKind kind, MatrixD& A,
              Vector<double, VectFull, CudaAlloc<double> >& x,
              const Vector<double, VectFull, CudaAlloc<double> >& b,
              P& M, Iteration<Titer>& iter)
    {
      return Dispatch<PrecondTraits<P>::native>::Run(kind, A, x, b, M, iter);
    }
  }


  //! Preconditioned CG on the GPU (Cg.cxx:45-116).
  template <class Titer, class Prop, class Preconditioner>
  int Cg(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
         Vector<double, VectFull, CudaAlloc<double> >& x,
         const Vector<double, VectFull, CudaAlloc<double> >& b,
         Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kCg, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int Cg(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
         Vector<double, VectFull, CudaAlloc<double> >& x,
         const Vector<double, VectFull, CudaAlloc<double> >& b,
         Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kCg, A, x, b, M, iter);
  }

  //! BiCGSTAB on the GPU (BiCgStab.cxx:43-145).
  template <class Titer, class Prop, class Preconditioner>
  int BiCgStab(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
               Vector<double, VectFull, CudaAlloc<double> >& x,
               const Vector<double, VectFull, CudaAlloc<double> >& b,
               Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kBiCgStab, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int BiCgStab(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
               Vector<double, VectFull, CudaAlloc<double> >& x,
               const Vector<double, VectFull, CudaAlloc<double> >& b,
               Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kBiCgStab, A, x, b, M, iter);
  }

  //! Conjugate gradient squared on the GPU (Cgs.cxx:45-132).
  template <class Titer, class Prop, class Preconditioner>
  int Cgs(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
          Vector<double, VectFull, CudaAlloc<double> >& x,
          const Vector<double, VectFull, CudaAlloc<double> >& b,
          Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kCgs, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int Cgs(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
          Vector<double, VectFull, CudaAlloc<double> >& x,
          const Vector<double, VectFull, CudaAlloc<double> >& b,
          Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kCgs, A, x, b, M, iter);
  }

  //! Transpose-free QMR on the GPU (TfQmr.cxx:44-243).
  template <class Titer, class Prop, class Preconditioner>
  int TfQmr(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
            Vector<double, VectFull, CudaAlloc<double> >& x,
            const Vector<double, VectFull, CudaAlloc<double> >& b,
            Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kTfQmr, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int TfQmr(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
            Vector<double, VectFull, CudaAlloc<double> >& x,
            const Vector<double, VectFull, CudaAlloc<double> >& b,
            Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kTfQmr, A, x, b, M, iter);
  }

  //! MINRES on the GPU (MinRes.cxx:46-153).
  template <class Titer, class Prop, class Preconditioner>
  int MinRes(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
             Vector<double, VectFull, CudaAlloc<double> >& x,
             const Vector<double, VectFull, CudaAlloc<double> >& b,
             Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kMinRes, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int MinRes(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
             Vector<double, VectFull, CudaAlloc<double> >& x,
             const Vector<double, VectFull, CudaAlloc<double> >& b,
             Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kMinRes, A, x, b, M, iter);
  }

  //! Restarted generalized conjugate residuals on the GPU (Gcr.cxx:45-141).
  template <class Titer, class Prop, class Preconditioner>
  int Gcr(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
          Vector<double, VectFull, CudaAlloc<double> >& x,
          const Vector<double, VectFull, CudaAlloc<double> >& b,
          Preconditioner& M, Iteration<Titer>& outer)
  {
    return b200::Solve(b200::kGcr, A, x, b, M, outer);
  }

  template <class Titer, class Prop, class Preconditioner>
  int Gcr(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
          Vector<double, VectFull, CudaAlloc<double> >& x,
          const Vector<double, VectFull, CudaAlloc<double> >& b,
          Preconditioner& M, Iteration<Titer>& outer)
  {
    return b200::Solve(b200::kGcr, A, x, b, M, outer);
  }

  //! CoCg on the GPU (CoCg.cxx:45-116): Cg's steps in real arithmetic.
  template <class Titer, class Prop, class Preconditioner>
  int CoCg(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
           Vector<double, VectFull, CudaAlloc<double> >& x,
           const Vector<double, VectFull, CudaAlloc<double> >& b,
           Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kCoCg, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int CoCg(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
           Vector<double, VectFull, CudaAlloc<double> >& x,
           const Vector<double, VectFull, CudaAlloc<double> >& b,
           Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kCoCg, A, x, b, M, iter);
  }

  //! Symmlq on the GPU (Symmlq.cxx:45-161).
  template <class Titer, class Prop, class Preconditioner>
  int Symmlq(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
             Vector<double, VectFull, CudaAlloc<double> >& x,
             const Vector<double, VectFull, CudaAlloc<double> >& b,
             Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kSymmlq, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int Symmlq(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
             Vector<double, VectFull, CudaAlloc<double> >& x,
             const Vector<double, VectFull, CudaAlloc<double> >& b,
             Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kSymmlq, A, x, b, M, iter);
  }

  //! QMR for symmetric systems on the GPU (QmrSym.cxx:41-165).
  template <class Titer, class Prop, class Preconditioner>
  int QmrSym(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
             Vector<double, VectFull, CudaAlloc<double> >& x,
             const Vector<double, VectFull, CudaAlloc<double> >& b,
             Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kQmrSym, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int QmrSym(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
             Vector<double, VectFull, CudaAlloc<double> >& x,
             const Vector<double, VectFull, CudaAlloc<double> >& b,
             Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kQmrSym, A, x, b, M, iter);
  }

  //! Lsqr on the GPU (Lsqr.cxx:40-135); the preconditioner is not used.
  template <class Titer, class Prop, class Preconditioner>
  int Lsqr(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
           Vector<double, VectFull, CudaAlloc<double> >& x,
           const Vector<double, VectFull, CudaAlloc<double> >& b,
           Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kLsqr, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int Lsqr(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
           Vector<double, VectFull, CudaAlloc<double> >& x,
           const Vector<double, VectFull, CudaAlloc<double> >& b,
           Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kLsqr, A, x, b, M, iter);
  }

  //! Biconjugate conjugate residuals on the GPU (BiCgcr.cxx:44-118).
  template <class Titer, class Prop, class Preconditioner>
  int BiCgcr(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
             Vector<double, VectFull, CudaAlloc<double> >& x,
             const Vector<double, VectFull, CudaAlloc<double> >& b,
             Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kBiCgcr, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int BiCgcr(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
             Vector<double, VectFull, CudaAlloc<double> >& x,
             const Vector<double, VectFull, CudaAlloc<double> >& b,
             Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kBiCgcr, A, x, b, M, iter);
  }

  //! Cg on the normal equations on the GPU (Cgne.cxx:40-127).
  template <class Titer, class Prop, class Preconditioner>
  int Cgne(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
           Vector<double, VectFull, CudaAlloc<double> >& x,
           const Vector<double, VectFull, CudaAlloc<double> >& b,
           Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kCgne, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int Cgne(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
           Vector<double, VectFull, CudaAlloc<double> >& x,
           const Vector<double, VectFull, CudaAlloc<double> >& b,
           Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kCgne, A, x, b, M, iter);
  }

  //! Biconjugate gradients on the GPU (BiCg.cxx:46-134).
  template <class Titer, class Prop, class Preconditioner>
  int BiCg(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
           Vector<double, VectFull, CudaAlloc<double> >& x,
           const Vector<double, VectFull, CudaAlloc<double> >& b,
           Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kBiCg, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int BiCg(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
           Vector<double, VectFull, CudaAlloc<double> >& x,
           const Vector<double, VectFull, CudaAlloc<double> >& b,
           Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kBiCg, A, x, b, M, iter);
  }

  //! Cgs with quasi-minimal smoothing on the GPU (QCgs.cxx:46-165).
  template <class Titer, class Prop, class Preconditioner>
  int QCgs(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
           Vector<double, VectFull, CudaAlloc<double> >& x,
           const Vector<double, VectFull, CudaAlloc<double> >& b,
           Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kQCgs, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int QCgs(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
           Vector<double, VectFull, CudaAlloc<double> >& x,
           const Vector<double, VectFull, CudaAlloc<double> >& b,
           Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kQCgs, A, x, b, M, iter);
  }

  //! BiCGSTAB(l) on the GPU, l = iter.GetRestart() (BiCgStabl.cxx:43-180).
  template <class Titer, class Prop, class Preconditioner>
  int BiCgStabl(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
                Vector<double, VectFull, CudaAlloc<double> >& x,
                const Vector<double, VectFull, CudaAlloc<double> >& b,
                Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kBiCgStabl, A, x, b, M, iter);
  }

  template <class Titer, class Prop, class Preconditioner>
  int BiCgStabl(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
                Vector<double, VectFull, CudaAlloc<double> >& x,
                const Vector<double, VectFull, CudaAlloc<double> >& b,
                Preconditioner& M, Iteration<Titer>& iter)
  {
    return b200::Solve(b200::kBiCgStabl, A, x, b, M, iter);
  }

  //! Restarted left-preconditioned GMRES(m) on the GPU (Gmres.cxx:44-183).
  template <class Titer, class Prop, class Preconditioner>
  int Gmres(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
            Vector<double, VectFull, CudaAlloc<double> >& x,
            const Vector<double, VectFull, CudaAlloc<double> >& b,
            Preconditioner& M, Iteration<Titer>& outer)
  {
    return b200::Solve(b200::kGmres, A, x, b, M, outer);
  }

  template <class Titer, class Prop, class Preconditioner>
  int Gmres(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
            Vector<double, VectFull, CudaAlloc<double> >& x,
            const Vector<double, VectFull, CudaAlloc<double> >& b,
            Preconditioner& M, Iteration<Titer>& outer)
  {
    return b200::Solve(b200::kGmres, A, x, b, M, outer);
  }

  //! Gmres(m) with classical Gram-Schmidt applied twice in place of the
  //! reference's modified Gram-Schmidt loop (sb2_gmres_cgs2): a labelled
  //! variant with no counterpart in the reference, same restarts, rotations,
  //! stopping rule and Iteration state; identity or Jacobi preconditioner
  //! and restart <= 32 (SorPreconditioner, the ILUT preconditioner or a
  //! larger restart raise Error).  For a preconditioner class this header
  //! does not know, Seldon's own Gmres runs on the device types.
  template <class Titer, class Prop, class Preconditioner>
  int GmresCgs2(Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
                Vector<double, VectFull, CudaAlloc<double> >& x,
                const Vector<double, VectFull, CudaAlloc<double> >& b,
                Preconditioner& M, Iteration<Titer>& outer)
  {
    return b200::Solve(b200::kGmresCgs2, A, x, b, M, outer);
  }

  template <class Titer, class Prop, class Preconditioner>
  int GmresCgs2(Matrix<double, Prop, RowSymSparse, CudaAlloc<double> >& A,
                Vector<double, VectFull, CudaAlloc<double> >& x,
                const Vector<double, VectFull, CudaAlloc<double> >& b,
                Preconditioner& M, Iteration<Titer>& outer)
  {
    return b200::Solve(b200::kGmresCgs2, A, x, b, M, outer);
  }


  //////////////////////////////
  // HARWELL-BOEING FILES     //
  //////////////////////////////


#ifdef SELDON_FILE_MATRIX_SPARSE_IOMATRIXMARKET_CXX

  //! WriteHarwellBoeing (IOMatrixMarket.cxx:394-511) of a device matrix:
  //! Seldon's writer on a host copy, so the file is the same byte for byte.
  template <class Prop>
  void WriteHarwellBoeing(const Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A,
                          const string& file_name)
  {
    Matrix<double, General, RowSparse> h;
    A.CopyToHost(h);
    WriteHarwellBoeing(h, file_name);
  }

  //! ReadHarwellBoeing (IOMatrixMarket.cxx:45-329) into a device matrix:
  //! Seldon reads the compressed columns on the host, and the matrix is
  //! assembled by rows on the device.
  template <class Prop>
  void ReadHarwellBoeing(string filename, Matrix<double, Prop, RowSparse, CudaAlloc<double> >& A)
  {
    Matrix<double, General, ColSparse> C;
    ReadHarwellBoeing(filename, C);
    const int n = C.GetN(), nnz = C.GetDataSize();
    std::vector<int> rows(nnz), cols(nnz);
    for (int j = 0; j < n; j++)
      for (int k = C.GetPtr()[j]; k < C.GetPtr()[j + 1]; k++)
        {
          rows[k] = C.GetInd()[k];
          cols[k] = j;
        }
    A.Reallocate(C.GetM(), n);
    if (nnz > 0)
      A.AssembleHost(nnz, &rows[0], &cols[0], C.GetData(), 0);
  }

#endif


  ///////////////////////////////////////////
  // ILUT: SELDON'S FACTOR, APPLIED ON GPU //
  ///////////////////////////////////////////


#ifdef SELDON_FILE_ILUT_PRECONDITIONING_HXX

  namespace b200
  {
    //! Reads Seldon's factor and permutations out of IlutPreconditioning's
    //! protected members (pointers to members named in a derived class).
    template <class Alloc>
    struct IlutState: public IlutPreconditioning<double, double, Alloc>
    {
      typedef IlutPreconditioning<double, double, Alloc> base;
      static const Matrix<double, General, ArrayRowSparse, Alloc>& Unsym(const base& p)
      {
        return p.*(&IlutState::mat_unsym);
      }
      static const Matrix<double, Symmetric, ArrayRowSymSparse, Alloc>& Sym(const base& p)
      {
        return p.*(&IlutState::mat_sym);
      }
      static const IVect& RowPerm(const base& p)
      {
        return p.*(&IlutState::permutation_row);
      }
      static const IVect& ColPerm(const base& p)
      {
        return p.*(&IlutState::permutation_col);
      }
    };
  }


  //! IlutPreconditioning whose Solve / TransSolve run on the device
  //! (IlutPreconditioning.cxx:329-374).  The factorization is Seldon's own:
  //! parameters and FactorizeMatrix go to a host IlutPreconditioning (GetIlut
  //! on the CPU, as in the reference), and the factor is then copied to the
  //! GPU, where the triangular sweeps reproduce SolveLU bit for bit.  Device
  //! matrices given to FactorizeMatrix are read back first.
  template <>
  class IlutPreconditioning<double, double, CudaAlloc<double> >
  {
  public:
    typedef IlutPreconditioning<double, double> host_type;
    typedef Vector<double, VectFull, CudaAlloc<double> > vector_type;

    enum {ILUT, ILU_D, ILUT_K, ILU_0, MILU_0, ILU_K};

  protected:
    host_type host_;
    bool symmetric_;
    sb2_precond* M_;

  public:
    IlutPreconditioning(): symmetric_(false), M_(0) {}
    ~IlutPreconditioning()
    {
      if (M_)
        sb2_precond_destroy(M_);
    }

    void Clear()
    {
      host_.Clear();
      if (M_)
        sb2_precond_destroy(M_);
      M_ = 0;
    }

    int GetFactorisationType() const { return host_.GetFactorisationType(); }
    int GetFillLevel() const { return host_.GetFillLevel(); }
    int GetAdditionalFillNumber() const { return host_.GetAdditionalFillNumber(); }
    int GetPrintLevel() const { return host_.GetPrintLevel(); }
    int GetPivotBlockInteger() const { return host_.GetPivotBlockInteger(); }
    double GetDroppingThreshold() const { return host_.GetDroppingThreshold(); }
    double GetDiagonalCoefficient() const { return host_.GetDiagonalCoefficient(); }
    double GetPivotThreshold() const { return host_.GetPivotThreshold(); }

    void SetFactorisationType(int t) { host_.SetFactorisationType(t); }
    void SetFillLevel(int k) { host_.SetFillLevel(k); }
    void SetAdditionalFillNumber(int k) { host_.SetAdditionalFillNumber(k); }
    void SetPrintLevel(int k) { host_.SetPrintLevel(k); }
    void SetPivotBlockInteger(int k) { host_.SetPivotBlockInteger(k); }
    void SetDroppingThreshold(double t) { host_.SetDroppingThreshold(t); }
    void SetDiagonalCoefficient(double a) { host_.SetDiagonalCoefficient(a); }
    void SetPivotThreshold(double t) { host_.SetPivotThreshold(t); }
    void SetSymmetricAlgorithm()
    {
      host_.SetSymmetricAlgorithm();
      symmetric_ = true;
    }
    void SetUnsymmetricAlgorithm()
    {
      host_.SetUnsymmetricAlgorithm();
      symmetric_ = false;
    }

    //! Seldon's factorization of a host matrix, then the upload.
    template <class Prop0, class Storage0, class Allocator0>
    void FactorizeMatrix(const IVect& perm, Matrix<double, Prop0, Storage0, Allocator0>& mat,
                         bool keep_matrix = false)
    {
      FactorizeHost(perm, mat, keep_matrix);
      Upload();
    }

    //! Device matrices are read back and factorized on the host.
    template <class Prop0>
    void FactorizeMatrix(const IVect& perm,
                         Matrix<double, Prop0, RowSparse, CudaAlloc<double> >& mat,
                         bool keep_matrix = false)
    {
      Matrix<double, General, RowSparse> h;
      mat.CopyToHost(h);
      FactorizeMatrix(perm, h, false);
      if (!keep_matrix)
        mat.Clear();
    }

    template <class Prop0>
    void FactorizeMatrix(const IVect& perm,
                         Matrix<double, Prop0, RowSymSparse, CudaAlloc<double> >& mat,
                         bool keep_matrix = false)
    {
      Matrix<double, Symmetric, RowSymSparse> h;
      mat.CopyToHost(h);
      FactorizeMatrix(perm, h, false);
      if (!keep_matrix)
        mat.Clear();
    }

    //! Library handle of the device factor.
    sb2_precond* GetHandle() const
    {
      if (!M_)
        throw WrongArgument("IlutPreconditioning", "no factor: call FactorizeMatrix first");
      return M_;
    }

    template <class Matrix1>
    void Solve(const Matrix1&, const vector_type& r, vector_type& z)
    {
      Apply(false, r, z);
    }

    template <class Matrix1>
    void TransSolve(const Matrix1&, const vector_type& r, vector_type& z)
    {
      Apply(true, r, z);
    }

    void Solve(vector_type& z)
    {
      vector_type r(z);
      Apply(false, r, z);
    }

    void TransSolve(vector_type& z)
    {
      vector_type r(z);
      Apply(true, r, z);
    }

    template <class TransStatus>
    void Solve(const TransStatus& transA, vector_type& z)
    {
      if (transA.Trans())
        TransSolve(z);
      else
        Solve(z);
    }

  protected:
    template <class Storage0, class Allocator0>
    void FactorizeHost(const IVect& perm, Matrix<double, General, Storage0, Allocator0>& mat,
                       bool keep_matrix)
    {
      if (symmetric_)
        throw Undefined("IlutPreconditioning::FactorizeMatrix",
                        "the symmetric algorithm needs symmetric storage");
      host_.FactorizeMatrix(perm, mat, keep_matrix);
    }

    // The unsymmetric algorithm on symmetric storage does not compile in the
    // reference (no Copy from RowSymSparse to ArrayRowSparse): only the
    // symmetric algorithm is offered for it.
    template <class Storage0, class Allocator0>
    void FactorizeHost(const IVect& perm, Matrix<double, Symmetric, Storage0, Allocator0>& mat,
                       bool keep_matrix)
    {
      if (!symmetric_)
        throw Undefined("IlutPreconditioning::FactorizeMatrix",
                        "symmetric storage needs SetSymmetricAlgorithm()");
      host_.FactorizeSymMatrix(perm, mat, keep_matrix);
    }

    void Upload()
    {
      typedef b200::IlutState<SELDON_DEFAULT_ALLOCATOR<double> > state;
      std::vector<int> fptr(1, 0), find;
      std::vector<double> fval;
      int n;
      if (symmetric_)
        {
          const Matrix<double, Symmetric, ArrayRowSymSparse>& F = state::Sym(host_);
          n = F.GetM();
          for (int i = 0; i < n; i++)
            {
              for (int k = 0; k < F.GetRowSize(i); k++)
                {
                  // position 0 holds 1/D(i); its index is never read
                  find.push_back(k == 0 ? i : F.Index(i, k));
                  fval.push_back(F.Value(i, k));
                }
              fptr.push_back(int(find.size()));
            }
        }
      else
        {
          const Matrix<double, General, ArrayRowSparse>& F = state::Unsym(host_);
          n = F.GetM();
          for (int i = 0; i < n; i++)
            {
              for (int k = 0; k < F.GetRowSize(i); k++)
                {
                  find.push_back(F.Index(i, k));
                  fval.push_back(F.Value(i, k));
                }
              fptr.push_back(int(find.size()));
            }
        }
      const IVect& pr = state::RowPerm(host_);
      const IVect& pc = symmetric_ ? pr : state::ColPerm(host_);
      std::vector<int> prow(n), pcol(n);
      for (int i = 0; i < n; i++)
        {
          prow[i] = pr(i);
          pcol[i] = pc(i);
        }
      sb2_precond* M = 0;
      b200::Check(sb2_precond_create_ilut(NULL, n, &fptr[0], find.empty() ? NULL : &find[0],
                                          fval.empty() ? NULL : &fval[0],
                                          n ? &prow[0] : NULL, n ? &pcol[0] : NULL,
                                          symmetric_ ? 1 : 0, &M),
                  "IlutPreconditioning::FactorizeMatrix");
      if (M_)
        sb2_precond_destroy(M_);
      M_ = M;
    }

    void Apply(bool trans, const vector_type& r, vector_type& z)
    {
      if (z.GetM() != r.GetM())
        z.Reallocate(r.GetM());
      b200::Check(trans ? sb2_precond_trans_solve(GetHandle(), r.GetData(), z.GetData(),
                                                  b200::GetStream())
                        : sb2_precond_solve(GetHandle(), r.GetData(), z.GetData(),
                                            b200::GetStream()),
                  trans ? "IlutPreconditioning::TransSolve" : "IlutPreconditioning::Solve");
    }
  };


  namespace b200
  {
    //! The library's Krylov drivers take the device factor directly.
    template <>
    struct PrecondTraits<IlutPreconditioning<double, double, CudaAlloc<double> > >
    {
      static const bool native = true;
      template <class MatrixD>
      static void Acquire(IlutPreconditioning<double, double, CudaAlloc<double> >& M,
                          const MatrixD&, PrecondHandle& h)
      {
        h.use = M.GetHandle();
      }
    };
  }

#endif

} // namespace Seldon.

#endif
