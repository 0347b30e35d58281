/* Minimal stand-in for <libusb-1.0/libusb.h>: the reference header only needs
 * these three type names to declare its USB device struct. No libusb function
 * is called by the oracle build (device code is not compiled). */
#ifndef ORACLE_LIBUSB_STUB_H
#define ORACLE_LIBUSB_STUB_H
typedef struct libusb_context libusb_context;
typedef struct libusb_device_handle libusb_device_handle;
struct libusb_transfer;
#endif
