"""Python side of the B200 AP-Cloud gravity step: ctypes binding of the C ABI
(``binding``), seeded initial conditions (``ics``) and the Controller step
sequence (``controller``)."""
